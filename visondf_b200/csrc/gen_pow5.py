"""Writes vdf_pow5.inc: 128-bit truncations of the powers of five 5^q,
q in [-342, 308], used by the decimal-to-double conversion in vdf_decimal.cuh.

Entry q holds F (hi, lo 64-bit halves) and e with 5^q = F_true * 2^e,
F_true in [2^127, 2^128) and F = floor(F_true): exact for 0 <= q <= 55, a
truncation (F <= F_true < F + 1) otherwise.  Exact integer arithmetic only.

Run: python visondf_b200/csrc/gen_pow5.py  (rewrites the .inc beside it).
"""
from pathlib import Path

QMIN, QMAX = -342, 308


def entry(q: int) -> tuple[int, int]:
    if q >= 0:
        v = 5 ** q
        b = v.bit_length()
        f = v << (128 - b) if b <= 128 else v >> (b - 128)
        return f, b - 128
    d = 5 ** (-q)
    b = d.bit_length()
    f = (1 << (127 + b)) // d
    return f, -(127 + b)


def main() -> None:
    his, los, es = [], [], []
    for q in range(QMIN, QMAX + 1):
        f, e = entry(q)
        assert (1 << 127) <= f < (1 << 128), q
        his.append(f >> 64)
        los.append(f & ((1 << 64) - 1))
        es.append(e)

    def rows(vals, fmt, per):
        out = []
        for i in range(0, len(vals), per):
            out.append("    " + ", ".join(fmt(v) for v in vals[i:i + per]) + ",")
        return "\n".join(out)

    text = (
        "// Generated by gen_pow5.py: 5^q = F * 2^e, F in [2^127, 2^128) truncated,\n"
        f"// q in [{QMIN}, {QMAX}].  Do not edit.\n"
        f"#define VDF_POW5_QMIN ({QMIN})\n"
        f"#define VDF_POW5_QMAX ({QMAX})\n"
        "#define VDF_POW5_HI_DATA \\\n" + rows(his, lambda v: f"0x{v:016x}ull", 4).replace("\n", " \\\n") + "\n"
        "#define VDF_POW5_LO_DATA \\\n" + rows(los, lambda v: f"0x{v:016x}ull", 4).replace("\n", " \\\n") + "\n"
        "#define VDF_POW5_E_DATA \\\n" + rows(es, str, 16).replace("\n", " \\\n") + "\n"
    )
    Path(__file__).with_name("vdf_pow5.inc").write_text(text)


if __name__ == "__main__":
    main()
