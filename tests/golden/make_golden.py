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

Run here, where the reference tree exists:  python tests/golden/make_golden.py
"""
from __future__ import annotations

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


def main():
    if not ob.ref_available():
        sys.exit("oracle/_ref/libvdf_ref.so missing: run `make -C oracle ref` where the reference tree exists")
    (HERE / "internals_sort_by.json").write_text(json.dumps(INTERNALS, indent=1) + "\n")
    np.savez_compressed(HERE / "ref_sort_cases.npz", **make_sort_cases())
    (HERE / "ref_groupby_cases.json").write_text(json.dumps(make_groupby_cases(), indent=1) + "\n")
    print("written:", sorted(p.name for p in HERE.iterdir()))


if __name__ == "__main__":
    main()
