"""Seeded synthetic CSV files for the ingest tests and benchmark: a header,
then rows mixing the column kinds read_csv infers -- decimals with a '.'
('d'), unsigned integers ('u'), 0/1 flags ('b'), quoted and bare strings
('s'), one-byte codes ('c') -- with optional CR LF line ends, empty fields
and a final record without terminator."""
from __future__ import annotations

import numpy as np

KINDS = ("d", "u", "b", "s", "c")


def _dec(rng, n, style):
    if style == 0:   # money-like: 2 decimals
        return [f"{x:.2f}" for x in rng.uniform(0, 5000, n)]
    if style == 1:   # full round-trip precision
        return [repr(float(x)) if "." in repr(float(x)) else repr(float(x)) + ".0"
                for x in rng.standard_normal(n) * 10.0 ** rng.integers(-8, 9, n)]
    if style == 2:   # exponents
        return [f"{m:.{p}f}e{e}" for m, p, e in zip(rng.uniform(1, 10, n), rng.integers(1, 18, n),
                                                    rng.integers(-320, 309, n))]
    # long mantissas (more than 19 significant digits)
    return ["".join(map(str, rng.integers(0, 10, int(k)))) + "." + "".join(map(str, rng.integers(0, 10, 5)))
            for k in rng.integers(15, 30, n)]


def make_csv(seed: int, nrow: int, kinds=None, crlf=False, empty_frac=0.0, quote="'", delim=",",
             trailing_newline=True, header=True, dec_style=None) -> bytes:
    rng = np.random.default_rng(seed)
    if kinds is None:
        kinds = [KINDS[i % len(KINDS)] for i in range(int(rng.integers(3, 9)))]
    cols = []
    for k in kinds:
        if k == "d":
            v = _dec(rng, nrow, int(rng.integers(0, 4)) if dec_style is None else dec_style)
            if nrow:
                v[0] = f"{float(rng.uniform(0, 100)):.3f}"   # a dotted number first: column reads 'd'
        elif k == "u":
            v = [str(int(x)) for x in rng.integers(0, 2 ** 32 if rng.random() < 0.5 else 10000, nrow)]
        elif k == "b":
            v = [str(int(x)) for x in rng.integers(0, 2, nrow)]
        elif k == "c":
            v = [chr(int(x)) for x in rng.integers(ord("A"), ord("Z") + 1, nrow)]
        else:
            words = ["alpha", "beta", "gamma", "delta x", f"{quote}in{delim} quotes{quote}", "N/A", "-5", "3.5.1"]
            v = [words[int(x)] for x in rng.integers(0, len(words), nrow)]
            if nrow:
                v[0] = "name"
        if empty_frac and nrow > 10:
            for i in np.nonzero(rng.random(nrow) < empty_frac)[0]:
                if i >= 10:   # keep the first 10 values so the inferred type is the intended one
                    v[int(i)] = ""
        cols.append(v)
    eol = "\r\n" if crlf else "\n"
    lines = []
    if header:
        lines.append(delim.join(f"col{j}_{k}" for j, k in enumerate(kinds)))
    for r in range(nrow):
        lines.append(delim.join(c[r] for c in cols))
    text = eol.join(lines)
    if trailing_newline and lines:
        text += eol
    return text.encode("latin-1")


def soup_csv(seed: int, nrow: int, ncol: int, quote="'", delim=",", short_row: int = -1) -> bytes:
    """Records whose fields mix plain text, fully quoted text and quotes in
    the middle of a field, with delimiters, CR, LF and CR LF inside the quoted
    parts, empty fields, and LF / CR LF / CR line ends chosen per record.  A
    header row of names comes first.  `short_row` >= 0 gives that record one
    field too few (a "column number problem")."""
    rng = np.random.default_rng(seed)
    plain = list("abcxyz 0123456789.-")
    inner = plain + [delim, "\n", "\r", "\r\n", delim + delim]

    def text(pool, k):
        return "".join(pool[int(i)] for i in rng.integers(0, len(pool), k))

    def field():
        kind = int(rng.integers(0, 5))
        if kind == 0:
            return ""
        if kind == 1:
            return text(plain, int(rng.integers(1, 8)))
        if kind == 2:
            return quote + text(inner, int(rng.integers(0, 10))) + quote
        if kind == 3:   # a quoted part in the middle of the field
            return text(plain, int(rng.integers(0, 3))) + quote + text(inner, int(rng.integers(0, 6))) + quote + \
                text(plain, int(rng.integers(0, 3)))
        return str(int(rng.integers(0, 100000)))

    eols = ["\n", "\r\n", "\r"]
    out = [delim.join(f"h{j}" for j in range(ncol)) + "\n"]
    for r in range(nrow):
        k = ncol - 1 if r == short_row else ncol
        out.append(delim.join(field() for _ in range(k)) + eols[int(rng.integers(0, 3))])
    return "".join(out).encode("latin-1")
