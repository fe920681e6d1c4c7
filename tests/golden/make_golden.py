"""Generates the golden fixtures in this directory.

  internals_sort_by.json  the reference documentation's own sort_by example
                          (V/INTERNALS.doc:1554-1632), transcribed: a 15-row
                          frame sorted by column n=2 ascending (sort_by(n)) and
                          descending (sort_by<0>(n)).
  ref_sort_cases.npz      seeded key columns and the permutations produced by
                          the REFERENCE'S OWN radix kernels
                          (radix_sort_uint{32,64}[_mt], built from the reference
                          sources by oracle/Makefile into oracle/_ref/), for
                          ascending order and for the reference code's
                          descending order (ascending + std::reverse).
  ref_groupby_cases.json  group counts and checksums (sum of counts, sum of each
                          value column's group sums) of the restated reference
                          hash group-by (ankerl map + simd_hash from the
                          reference tree) on seeded frames.
  ref_csv_cases.npz       CSV inputs (seeded synthetic files from
                          tests/csv_gen.py plus hand-written edge cases) and the
                          tables the REFERENCE'S OWN record parser and
                          fast_float produce for them (oracle/_ref shim,
                          ref_csv_read), in the oracle's blob layout; `meta`
                          holds each case's delimiter, quote and header flag.

Run here, where the reference tree exists:  python tests/golden/make_golden.py
(`python tests/golden/make_golden.py csv` rewrites only ref_csv_cases.npz)
"""
from __future__ import annotations

import ctypes as C
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parent.parent))

import oracle_bind as ob  # noqa: E402
from visondf_b200 import datagen  # noqa: E402  (numpy only; does not need the GPU library)

INTERNALS = {
    "source": "V/INTERNALS.doc:1554-1632 (Dataframe.sort_by example)",
    "columns": {
        "col1": ["id1", "id2", "id3", "id4", "id5", "id6", "id7", "id8", "id9", "id10", "id11", "id12", "id13",
                 "id14", "id15"],
        "col2": [1, 6, 1, 6, 1, 6, 1, 6, 6, 1, 6, 6, 6, 1, 16],
        "col3": [2, 7, 2, 7, 2, 7, 2, 7, 7, 2, 7, 7, 7, 2, 7],
        "col4": [3, 8, 3, 8, 3, 8, 3, 8, 8, 3, 8, 8, 8, 3, 8],
        "col5": ["aa", "bb", "cc", "uu", "s4", "s9", "a4", "m9", "s9", "a4", "m9", "m9", "s9", "NA", "m9"],
    },
    "types": {"col1": "str", "col2": "uint", "col3": "uint", "col4": "uint", "col5": "str"},
    "sort_col_index": 2,
    "asc_col1": ["id1", "id3", "id5", "id7", "id10", "id14", "id2", "id4", "id6", "id8", "id9", "id11", "id12",
                 "id13", "id15"],
    "desc_col1": ["id2", "id4", "id6", "id8", "id9", "id11", "id12", "id13", "id15", "id1", "id3", "id5", "id7",
                  "id10", "id14"],
}

SINGLE_DTYPES = [np.int32, np.int64, np.uint32, np.uint64, np.float64]
SIZES = [1, 33, 1500]
DISTS = ["uniform", "few", "sorted"]


def make_sort_cases() -> dict:
    out = {}
    rng = np.random.default_rng(0xB200 + 999)
    case = 0
    for dt in SINGLE_DTYPES:
        for n in SIZES:
            for dist in DISTS:
                k = datagen.keys_for(dist, dt, n, rng)
                p_asc, _ = ob.ref_sort([k], ob.ASC, cores=1)
                p_asc4, _ = ob.ref_sort([k], ob.ASC, cores=4)
                assert (p_asc == p_asc4).all()
                p_rev, _ = ob.ref_sort([k], ob.DESC_REVERSE, cores=1)
                out[f"c{case}_k0"] = k
                out[f"c{case}_asc"] = p_asc
                out[f"c{case}_rev"] = p_rev
                case += 1
    multi = [
        ([np.int64, np.int32], 3000, ["few", "zipf"]),
        ([np.int32, np.int64, np.uint32], 2000, ["small", "few", "uniform"]),
        ([np.float64, np.uint64], 1000, ["few", "small"]),
    ]
    for dts, n, dists in multi:
        ks = [datagen.keys_for(d, t, n, rng) for t, d in zip(dts, dists)]
        p_asc, _ = ob.ref_sort(ks, ob.ASC, cores=1)
        p_rev, _ = ob.ref_sort(ks, ob.DESC_REVERSE, cores=2)
        for i, k in enumerate(ks):
            out[f"c{case}_k{i}"] = k
        out[f"c{case}_asc"] = p_asc
        out[f"c{case}_rev"] = p_rev
        case += 1
    out["n_cases"] = np.array([case])
    return out


def make_groupby_cases() -> list:
    cases = []
    for seed, n, distinct, kdt in [(1, 5000, 40, np.int32), (2, 20000, 5000, np.int64), (3, 777, 1, np.int32),
                                   (4, 3000, 3000, np.int64)]:
        rng = np.random.default_rng(0xB200 + 500 + seed)
        pool = datagen.distinct_pool(rng, distinct, kdt)
        key = pool[rng.integers(0, distinct, size=n)]
        v1 = np.round(rng.standard_normal(n) * 1000) / 8.0  # exactly representable sums
        v2 = rng.integers(-10**9, 10**9, size=n, dtype=np.int64)
        g, chk = ob.ref_groupby([key], [v1, v2], cores=1)
        g4, chk4 = ob.ref_groupby([key], [v1, v2], cores=4)
        assert g == g4
        cases.append({"seed": seed, "n": n, "distinct": distinct, "key_dtype": np.dtype(kdt).name,
                      "n_groups": g, "sum_count": chk[0], "sum_v1": chk[1], "sum_v2": chk[2]})
    return cases


def hard_decimals(seed: int, count: int) -> list:
    """Decimal strings at and next to the exact halfway points between
    adjacent doubles (exact rational arithmetic), plus out-of-range values."""
    import math
    import random
    import struct
    from fractions import Fraction

    def exact(fr):
        k = fr.denominator.bit_length() - 1
        assert fr.denominator == 1 << k
        digits = str(fr.numerator * 5 ** k)
        if k == 0:
            return digits
        if len(digits) <= k:
            digits = "0" * (k - len(digits) + 1) + digits
        return digits[:-k] + "." + digits[-k:]

    rnd = random.Random(seed)
    out = ["0.5", "1e400", "-1e400", "1e-400", "2.4703282292062327e-324", "2.4703282292062328e-324",
           "4.9e-324", "1.7976931348623158e308", "1.7976931348623159e308", "nan", "-inf", "Infinity", "NA",
           "-0.0", "12abc", "1e", "1e+", ".5", "-.5", "5."]
    while len(out) < count:
        b = rnd.getrandbits(63) if rnd.random() < 0.8 else rnd.getrandbits(52)
        x = struct.unpack("<d", struct.pack("<Q", b))[0]
        y = math.nextafter(x, math.inf)
        if not (0 < x and math.isfinite(y)):
            continue
        h = (Fraction(x) + Fraction(y)) / 2
        s = exact(h)
        out += [s, s + "000000000000000000001", exact(h - Fraction(1, 1 << 1100)) if h > Fraction(1, 1 << 1100) else s]
    return out[:count]


def make_csv_cases() -> dict:
    import csv_gen
    cases = []
    for seed in range(10):
        cases.append(dict(data=csv_gen.make_csv(100 + seed, 40 + 23 * seed, crlf=seed % 3 == 1,
                                                empty_frac=0.05 * (seed % 2), header=seed % 4 != 3,
                                                trailing_newline=seed % 5 != 4, quote="'" if seed % 2 else '"'),
                          delim=",", quote="'" if seed % 2 else '"', header=seed % 4 != 3))
    cases.append(dict(data=csv_gen.make_csv(7, 300, kinds=["d"] * 4, dec_style=2), delim=",", quote="'",
                      header=True))
    cases.append(dict(data=("x\n" + "\n".join(hard_decimals(11, 600)) + "\n").encode(), delim=",", quote="'",
                      header=True))
    edge = [
        (b"a;b;c\n1;'x;y';2.5\n3;'multi\nline';4.0\n", ";", "'", True),   # quoted delimiter and LF
        (b"a,b\r1,2\r3,4\r", ",", "'", True),                             # CR-only line ends
        (b"1,2,x\r\n3,4,y\r\n", ",", "'", False),                           # no header, CR LF: first row keeps the CR
        (b",2,\n3,,5\n", ",", "'", False),                                # no header, empty first-line fields
        (b"h1,h2\n", ",", "'", True),                                      # header only
        (b"h1,h2\n1,2\n3\n4,5\n", ",", "'", True),                         # a record with fewer fields
        (b"n\n0\n1\n1\n0\n7\n-3\n", ",", "'", True),                         # 0/1 flags read as 'b'
        (b"n\n4294967295\n4294967296\n0012\n7\n", ",", "'", True),          # u32 limits
        (b"n\n1\n2\n3\n4\n5\n6\n7\n8\n9\n10\n12x\n\n-5\n+5\n", ",", "'", True),  # 'u' past the first 10
        (b"c\nA\nB\nC", ",", "'", True),                                   # one-byte codes, no final LF
        (b"c\nA\nB\n\nC", ",", "'", True),                                 # an empty record reads "NA" ('s')
        (b"v\n1.5\nnan\n-nan\ninf\n-Infinity\n1e999\n1e-999\n+1\n 2\n", ",", "'", True),
    ]
    for data, d, q, h in edge:
        cases.append(dict(data=data, delim=d, quote=q, header=h))
    out, meta = {}, []
    for i, c in enumerate(cases):
        r = ob.ref_csv_read(c["data"], delim=c["delim"], header=c["header"], quote=c["quote"])
        size = C.c_size_t(0)
        lib = ob.ref()
        blob = lib.ref_csv_read(c["data"], len(c["data"]), c["delim"].encode(), 1 if c["header"] else 0,
                                c["quote"].encode(), 1, C.byref(size), None)
        raw = C.string_at(blob, size.value)
        lib.ref_csv_free(blob)
        assert r.nrow == ob.CsvResult(raw).nrow
        out[f"csv{i}"] = np.frombuffer(c["data"], dtype=np.uint8)
        out[f"blob{i}"] = np.frombuffer(raw, dtype=np.uint8)
        meta.append(dict(delim=c["delim"], quote=c["quote"], header=c["header"]))
    out["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    return out


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "csv":
        np.savez_compressed(HERE / "ref_csv_cases.npz", **make_csv_cases())
        print("written: ref_csv_cases.npz")
        return
    if not ob.ref_available():
        sys.exit("oracle/_ref/libvdf_ref.so missing: run `make -C oracle ref` where the reference tree exists")
    (HERE / "internals_sort_by.json").write_text(json.dumps(INTERNALS, indent=1) + "\n")
    np.savez_compressed(HERE / "ref_sort_cases.npz", **make_sort_cases())
    (HERE / "ref_groupby_cases.json").write_text(json.dumps(make_groupby_cases(), indent=1) + "\n")
    np.savez_compressed(HERE / "ref_csv_cases.npz", **make_csv_cases())
    print("written:", sorted(p.name for p in HERE.iterdir()))


if __name__ == "__main__":
    main()
