"""The CPU oracle, pinned against the reference: its documentation example
(V/INTERNALS.doc:1554-1632), fixtures produced by the reference's own radix
kernels (tests/golden/ref_sort_cases.npz) and, where the reference shim is
built, live runs of those kernels.  No GPU needed."""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle_bind as ob
from visondf_b200 import datagen

GOLDEN = Path(__file__).resolve().parent / "golden"


def load_sort_cases():
    z = np.load(GOLDEN / "ref_sort_cases.npz")
    cases = []
    for c in range(int(z["n_cases"][0])):
        keys, i = [], 0
        while f"c{c}_k{i}" in z:
            keys.append(z[f"c{c}_k{i}"])
            i += 1
        cases.append((keys, z[f"c{c}_asc"], z[f"c{c}_rev"]))
    return cases


def internals_keys():
    d = json.loads((GOLDEN / "internals_sort_by.json").read_text())
    col = list(d["columns"])[d["sort_col_index"]]
    key = np.array(d["columns"][col], dtype=np.uint32)
    ids = np.array(d["columns"]["col1"])
    return d, key, ids


def test_internals_doc_example_ascending():
    d, key, ids = internals_keys()
    perm = ob.argsort([key], ob.ASC)
    assert list(ids[perm]) == d["asc_col1"]


def test_internals_doc_example_descending_is_stable():
    d, key, ids = internals_keys()
    perm = ob.argsort([key], ob.DESC_STABLE)
    assert list(ids[perm]) == d["desc_col1"]


def test_reference_code_descending_reverses_ties():
    # The reference code's descending sort is ascending + std::reverse
    # (sort_integers.inl:225-227): ties come out in reverse row order, unlike
    # the documented table.
    d, key, ids = internals_keys()
    perm = ob.argsort([key], ob.DESC_REVERSE)
    assert list(ids[perm]) == list(reversed(d["asc_col1"]))
    assert list(ids[perm]) != d["desc_col1"]


@pytest.mark.parametrize("case", range(len(load_sort_cases())))
def test_oracle_matches_reference_radix_fixtures(case):
    keys, p_asc, p_rev = load_sort_cases()[case]
    assert (ob.argsort(keys, ob.ASC) == p_asc).all()
    assert (ob.argsort(keys, ob.DESC_REVERSE) == p_rev).all()


@pytest.mark.parametrize("dt", [np.int32, np.int64, np.uint32, np.uint64, np.float64, np.float32])
@pytest.mark.parametrize("dist", ["uniform", "few", "equal", "reversed"])
def test_oracle_matches_numpy_stable(dt, dist):
    rng = np.random.default_rng(7)
    k = datagen.keys_for(dist, dt, 20011, rng)
    exp = np.argsort(k, kind="stable")
    if np.dtype(dt).kind == "f":
        # numpy orders -0.0 == +0.0 (stable) while the IEEE image orders -0.0 first
        exp = np.lexsort((np.arange(k.size), np.signbit(k) == 0, k)) if dist == "few" else exp
    assert (ob.argsort([k]) == exp).all()


def test_oracle_multikey_matches_lexsort():
    rng = np.random.default_rng(3)
    k1 = rng.integers(-5, 5, 50000).astype(np.int64)
    k2 = rng.integers(-3, 3, 50000).astype(np.int32)
    k3 = rng.integers(0, 4, 50000).astype(np.uint32)
    assert (ob.argsort([k1, k2, k3]) == np.lexsort((k3, k2, k1))).all()
    exp_desc = np.lexsort((-k3.astype(np.int64), -k2.astype(np.int64), -k1))
    assert (ob.argsort([k1, k2, k3], ob.DESC_STABLE) == exp_desc).all()


@pytest.mark.skipif(not ob.ref_available(), reason="reference shim not built (needs the reference tree)")
@pytest.mark.parametrize("seed", [11, 12])
def test_oracle_matches_live_reference(seed):
    rng = np.random.default_rng(seed)
    for dt in (np.int32, np.int64, np.uint64, np.float64):
        k = datagen.keys_for("zipf" if np.dtype(dt).kind != "f" else "uniform", dt, 100_003, rng)
        for cores in (1, 3, 8):
            p, _ = ob.ref_sort([k], ob.ASC, cores=cores)
            assert (ob.argsort([k]) == p).all()


def python_groupby(keys, vals):
    """Pure-Python restatement for small inputs: dict keyed by the key tuple."""
    groups = {}
    for r in range(keys[0].size):
        kt = tuple(k[r].item() for k in keys)
        groups.setdefault(kt, []).append(r)
    return groups


def test_oracle_groupby_matches_python():
    rng = np.random.default_rng(5)
    n = 3000
    k1 = rng.integers(-4, 4, n).astype(np.int32)
    k2 = rng.integers(0, 3, n).astype(np.int64)
    v1 = rng.standard_normal(n)
    v2 = rng.integers(-10**12, 10**12, n).astype(np.int64)
    og = ob.groupby([k1, k2], [v1, v2])
    pg = python_groupby([k1, k2], [v1, v2])
    assert og.n_groups == len(pg)
    order = sorted(pg, key=lambda t: (t[0], t[1]))
    for g, kt in enumerate(order):
        rows = pg[kt]
        assert (og.keys[0][g], og.keys[1][g]) == kt
        assert og.count[g] == len(rows)
        assert og.sum[1][g] == int(np.sum(v2[rows].astype(object)))
        assert og.min[1][g] == v2[rows].min() and og.max[1][g] == v2[rows].max()
        assert og.min[0][g] == v1[rows].min() and og.max[0][g] == v1[rows].max()
        exact = float(sum(map(__import__("fractions").Fraction, v1[rows])))
        assert abs(og.sum[0][g] - exact) <= 1e-15 * np.abs(v1[rows]).sum()
        assert og.mean[0][g] == pytest.approx(exact / len(rows), rel=1e-14, abs=1e-15)


def test_oracle_groupby_int128_sums():
    n = 1000
    key = np.zeros(n, np.int32)
    v = np.full(n, np.iinfo(np.int64).max, np.int64)
    og = ob.groupby([key], [v])
    exact = int(np.iinfo(np.int64).max) * n
    got = (int(og.sum_hi[0][0]) << 64) + (int(og.sum[0][0]) & ((1 << 64) - 1))
    assert got == exact


def test_oracle_groupby_matches_reference_checksums():
    cases = json.loads((GOLDEN / "ref_groupby_cases.json").read_text())
    for c in cases:
        rng = np.random.default_rng(0xB200 + 500 + c["seed"])
        pool = datagen.distinct_pool(rng, c["distinct"], np.dtype(c["key_dtype"]).type)
        key = pool[rng.integers(0, c["distinct"], size=c["n"])]
        v1 = np.round(rng.standard_normal(c["n"]) * 1000) / 8.0
        v2 = rng.integers(-10**9, 10**9, size=c["n"], dtype=np.int64)
        og = ob.groupby([key], [v1, v2])
        assert og.n_groups == c["n_groups"]
        assert og.count.sum() == c["sum_count"]
        assert og.sum[0].sum() == pytest.approx(c["sum_v1"], rel=1e-12)
        assert float(og.sum[1].sum()) == pytest.approx(c["sum_v2"], rel=1e-12)


def test_oracle_first_appearance_order():
    key = np.array([5, 3, 5, 9, 3, 1], np.int32)
    og = ob.groupby([key], [], sorted_groups=False)
    assert list(og.keys[0]) == [5, 3, 9, 1]  # the ankerl map's insertion order
    og = ob.groupby([key], [], sorted_groups=True)
    assert list(og.keys[0]) == [1, 3, 5, 9]


@pytest.mark.skipif(not ob.ref_available(), reason="reference shim not built (needs the reference tree)")
@pytest.mark.parametrize("cores", [1, 5])
def test_live_reference_groupby_multikey_checksums(cores):
    # composite (int64, int32) keys: 14 bytes with the reference's separators
    rng = np.random.default_rng(31)
    n = 60_000
    k1 = rng.integers(-3, 3, n).astype(np.int64)
    k2 = rng.integers(0, 1000, n).astype(np.int32)
    v1 = np.round(rng.standard_normal(n) * 1000) / 8.0
    v2 = rng.integers(-10**6, 10**6, n).astype(np.int32)
    g, chk = ob.ref_groupby([k1, k2], [v1, v2], cores=cores)
    og = ob.groupby([k1, k2], [v1, v2])
    assert g == og.n_groups
    assert chk[0] == og.count.sum()
    assert chk[1] == pytest.approx(og.sum[0].sum(), rel=1e-12)
    assert chk[2] == float(og.sum[1].sum())


def test_pivot_matches_the_documented_example():
    """INTERNALS.doc:1251-1296 (pivot of the 15-row frame): col key col5
    (A/B), row key the second col1 (D/C), values the second col3; the
    documented result is A: D=27, C=0 and B: D=14, C=30."""
    col5 = list("AAABBABBBAABBBB")
    col1b = list("DDCCCDCDDCDCDCD")
    col3b = np.array([3, 8, 0, 8, 3, 8, 3, 3, 8, 0, 8, 8, 0, 8, 3], np.float64)
    p = ob.pivot(col5, col1b, col3b)
    assert [col5[r] for r in p.colkey_row] == ["A", "B"]
    assert [col1b[r] for r in p.rowkey_row] == ["D", "C"]
    assert p.matrix.tolist() == [[27.0, 0.0], [14.0, 30.0]]


def test_pivot_oracle_against_a_dict_walk():
    rng = np.random.default_rng(5)
    n = 5000
    cols = [f"c{x}" for x in rng.integers(0, 37, n)]
    rows = ["r" * int(x % 3) + str(x) for x in rng.integers(0, 101, n)]
    for dt in (np.int32, np.uint32, np.int64, np.float64):
        vals = rng.integers(-1000, 1000, n).astype(dt) if dt != np.float64 else rng.standard_normal(n)
        p = ob.pivot(cols, rows, vals)
        ci, ri, acc = {}, {}, {}
        for c, r, v in zip(cols, rows, vals):
            ci.setdefault(c, len(ci))
            ri.setdefault(r, len(ri))
            acc[(c, r)] = acc.get((c, r), dt(0)) + v
        assert [cols[r] for r in p.colkey_row] == list(ci)
        assert [rows[r] for r in p.rowkey_row] == list(ri)
        exp = np.zeros((len(ci), len(ri)), vals.dtype)
        for (c, r), v in acc.items():
            exp[ci[c], ri[r]] = v
        assert (p.matrix == exp).all()
