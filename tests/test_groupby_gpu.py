"""GPU sort-based group-by through the C-ABI against the CPU oracle's hash
group-by (groups compared in ascending key order): keys, counts and integer
sum/min/max bit-exact; f64 sums and means within 1e-12."""
import numpy as np
import pytest
import torch

import oracle_bind as ob
import visondf_b200 as vdf
from gpu_util import assert_f64_close, bits_equal, dev, host
from visondf_b200 import datagen

pytestmark = pytest.mark.gpu


def compare(og, gr, vals, what=""):
    assert gr.n_groups == og.n_groups, f"{what}: groups {gr.n_groups} != {og.n_groups}"
    for a, b in zip(gr.keys, og.keys):
        assert bits_equal(host(a), b), f"{what}: group keys differ"
    assert (host(gr.count) == og.count).all()
    for v, (ga, ov) in enumerate(zip(gr.aggs, vals)):
        if ov.dtype.kind == "f":
            assert_f64_close(host(ga.sum), og.sum[v], og.abs[v], f"{what} sum[{v}]")
            assert_f64_close(host(ga.mean), og.mean[v], og.abs[v] / og.count, f"{what} mean[{v}]")
            assert bits_equal(host(ga.min), og.min[v]) and bits_equal(host(ga.max), og.max[v])
        else:
            assert (host(ga.sum) == og.sum[v]).all(), f"{what}: int sum lo"
            assert (host(ga.sum_hi) == og.sum_hi[v]).all(), f"{what}: int sum hi"
            assert bits_equal(host(ga.min), og.min[v]) and bits_equal(host(ga.max), og.max[v])
            np.testing.assert_allclose(host(ga.mean), og.mean[v], rtol=1e-12)


def frame(n, kdts, distinct, rng, vdts=(np.float64, np.int64)):
    keys = []
    for t in kdts:
        pool = datagen.distinct_pool(rng, distinct, t) if np.dtype(t).kind != "f" else rng.standard_normal(distinct)
        keys.append(pool[rng.integers(0, distinct, size=n)])
    vals = []
    for t in vdts:
        if np.dtype(t).kind == "f":
            vals.append(rng.standard_normal(n).astype(t))
        else:
            info = np.iinfo(t)
            vals.append(rng.integers(info.min, info.max, size=n, dtype=t, endpoint=True))
    return keys, vals


@pytest.mark.parametrize("n", [1, 2, 33, 1023, 1024, 1025, 4097, 100_000])
@pytest.mark.parametrize("distinct", [1, 7, 5000])
def test_sort_groupby_single_key(ctx, n, distinct):
    rng = np.random.default_rng(n + distinct)
    keys, vals = frame(n, [np.int32], distinct, rng)
    gr = ctx.sort_groupby([dev(k) for k in keys], [dev(v) for v in vals], agg_cols=[0, 1])
    compare(ob.groupby(keys, vals), gr, vals, f"n={n} d={distinct}")
    perm = ob.argsort(keys)
    assert (host(gr.perm).view(np.uint32) == perm).all()
    for v, p in zip(vals, gr.payload):
        assert bits_equal(host(p), v[perm])


@pytest.mark.parametrize("kdts", [(np.int64, np.int32), (np.int32, np.uint64, np.int32), (np.float64,),
                                  (np.uint32, np.uint32, np.uint32, np.uint32)])
def test_sort_groupby_multi_key(ctx, kdts):
    rng = np.random.default_rng(len(kdts))
    keys, vals = frame(300_007, kdts, 23, rng)
    gr = ctx.sort_groupby([dev(k) for k in keys], [dev(v) for v in vals], agg_cols=[0, 1])
    compare(ob.groupby(keys, vals), gr, vals, str(kdts))


@pytest.mark.parametrize("vdts", [(np.int32,), (np.uint64, np.float32), (np.uint32, np.int64, np.float64, np.int32),
                                  ()])
def test_value_types(ctx, vdts):
    rng = np.random.default_rng(77)
    keys, vals = frame(120_001, [np.int64], 300, rng, vdts)
    gr = ctx.sort_groupby([dev(k) for k in keys], [dev(v) for v in vals], agg_cols=list(range(len(vals))))
    compare(ob.groupby(keys, vals), gr, vals, str(vdts))


def test_long_segments_cross_many_tiles(ctx):
    # 90/10 skew over 16 keys: two segments of ~450k rows span hundreds of tiles
    rng = np.random.default_rng(5)
    n = 1_000_000
    pool = datagen.distinct_pool(rng, 16, np.int32)
    p = np.full(16, 0.10 / 14)
    p[:2] = 0.45
    key = pool[rng.choice(16, size=n, p=p)]
    v1 = np.exp(rng.standard_normal(n))
    v2 = rng.integers(0, 1 << 40, size=n, dtype=np.int64)
    gr = ctx.sort_groupby([dev(key)], [dev(v1), dev(v2)], agg_cols=[0, 1])
    og = ob.groupby([key], [v1, v2])
    compare(og, gr, [v1, v2], "skew")
    # same-sign data: the plain 1e-12 relative bound must hold too
    np.testing.assert_allclose(host(gr.aggs[0].sum), og.sum[0], rtol=1e-12)


@pytest.mark.parametrize("tail", [[1] * 300, [1] * 295 + [5]])
def test_tiles_of_single_row_groups_beside_scanned_tiles(ctx, tail):
    """Tiles (512 rows) where every row starts a group take a path without a
    scan; this places them next to tiles that scan, with a group crossing
    the first tile boundary, a group covering whole tiles, a whole-tile group
    ending exactly at a boundary before a single-row tile, and a last tile
    that is partial."""
    runs = [1] * 511 + [2] + [1] * 511 + [1] * 512 + [1500] + [1] * 36 + [512] + [1] * 512 + tail
    n = int(np.sum(runs))
    key = np.repeat(np.arange(len(runs), dtype=np.int64) * 3 - 1000, runs)
    rng = np.random.default_rng(21)
    v1 = rng.standard_normal(n)
    v2 = rng.integers(-2**62, 2**62, size=n, dtype=np.int64)
    og = ob.groupby([key], [v1, v2])
    gr = ctx.groupby_sorted([dev(key)], [dev(v1), dev(v2)], want_row_group=True, want_group_start=True)
    compare(og, gr, [v1, v2], "sorted mix")
    starts = np.concatenate([[0], np.cumsum(runs)[:-1]])
    assert (host(gr.group_start).view(np.uint32) == starts).all()
    assert (host(gr.row_group).view(np.uint32) == np.repeat(np.arange(len(runs)), runs)).all()
    shuffled = rng.permutation(n)
    gs = ctx.sort_groupby([dev(key[shuffled])], [dev(v1[shuffled]), dev(v2[shuffled])], agg_cols=[0, 1])
    compare(og, gs, [v1, v2], "shuffled mix")


@pytest.mark.parametrize("nkeys", [1, 2])
def test_tiles_of_mostly_single_row_groups(ctx, nkeys):
    """Tiles (512 rows) where at most 32 rows continue a group take a striped
    path: one-row groups written by consecutive lanes, the head row of a
    longer group walks it.  Runs of 2-3 rows, a 33-row group inside a tile, a
    group running over a tile boundary, one ending exactly at a boundary, one
    covering the first row of a tile, and a partial last tile."""
    rng = np.random.default_rng(31)
    runs = []
    while sum(runs) < 40_000:
        r = int(rng.choice([1, 2, 3], p=[0.97, 0.02, 0.01]))
        runs.append(r)
    runs += [1] * 100 + [33] + [1] * 500 + [7] + [1] * 300 + [2] * 3 + [1] * 77
    # a group spanning a tile boundary and one ending exactly at one
    csum = np.cumsum(runs)
    runs[int(np.searchsorted(csum, 30 * 512))] += 4
    n = int(np.sum(runs))
    gid = np.repeat(np.arange(len(runs), dtype=np.int64), runs)
    keys = [gid * 5 - 7] if nkeys == 1 else [(gid // 3).astype(np.int32), (gid % 3) * 11 - 4]
    v1 = rng.standard_normal(n)
    v2 = rng.integers(-2**40, 2**40, size=n, dtype=np.int64)
    og = ob.groupby(keys, [v1, v2])
    gr = ctx.groupby_sorted([dev(k) for k in keys], [dev(v1), dev(v2)], want_row_group=True,
                            want_group_start=True)
    compare(og, gr, [v1, v2], "mostly single rows")
    starts = np.concatenate([[0], np.cumsum(runs)[:-1]])
    assert (host(gr.group_start).view(np.uint32) == starts).all()
    assert (host(gr.row_group).view(np.uint32) == np.repeat(np.arange(len(runs)), runs)).all()
    shuffled = rng.permutation(n)
    gs = ctx.sort_groupby([dev(k[shuffled]) for k in keys], [dev(v1[shuffled]), dev(v2[shuffled])],
                          agg_cols=[0, 1])
    compare(og, gs, [v1, v2], "shuffled mostly single rows")


def test_int64_sum_overflow_is_exact(ctx):
    n = 300_000
    key = np.zeros(n, np.int64)
    key[n // 2:] = 1
    v = np.full(n, np.iinfo(np.int64).max - 5, np.int64)
    v[::3] = np.iinfo(np.int64).min + 2
    gr = ctx.sort_groupby([dev(key)], [dev(v)], agg_cols=[0])
    og = ob.groupby([key], [v])
    compare(og, gr, [v], "overflow")


def test_groupby_sorted_entry_and_row_group(ctx):
    rng = np.random.default_rng(8)
    keys, vals = frame(50_000, [np.int32, np.int64], 40, rng)
    perm = ob.argsort(keys)
    sk = [k[perm] for k in keys]
    sv = [v[perm] for v in vals]
    gr = ctx.groupby_sorted([dev(k) for k in sk], [dev(v) for v in sv], want_row_group=True, want_group_start=True)
    og = ob.groupby(keys, vals)
    compare(og, gr, vals, "sorted entry")
    rg = host(gr.row_group).view(np.uint32)
    gs = host(gr.group_start).view(np.uint32)
    assert rg[0] == 0 and rg[-1] == gr.n_groups - 1
    assert (np.diff(rg.astype(np.int64)) >= 0).all()
    assert (rg[gs] == np.arange(gr.n_groups)).all()


def test_transform_broadcast_matches_reference_semantics(ctx):
    # CreateValueCol: every original row receives its group's aggregate
    rng = np.random.default_rng(12)
    keys, vals = frame(40_000, [np.int32], 100, rng)
    gr = ctx.sort_groupby([dev(k) for k in keys], [dev(v) for v in vals], agg_cols=[0, 1], want_row_group=True)
    out = ctx.broadcast(gr.row_group, gr.count, perm=gr.perm)
    og = ob.groupby(keys, vals)
    lookup = {k: c for k, c in zip(og.keys[0].tolist(), og.count.tolist())}
    exp = np.array([lookup[k] for k in keys[0].tolist()])
    assert (host(out) == exp).all()


def test_descending_groups(ctx):
    rng = np.random.default_rng(14)
    keys, vals = frame(30_000, [np.int64], 50, rng)
    gr = ctx.sort_groupby([dev(k) for k in keys], [dev(v) for v in vals], agg_cols=[0, 1],
                          order=vdf.ORDER_DESC_STABLE)
    og = ob.groupby(keys, vals)
    assert (host(gr.keys[0]) == og.keys[0][::-1]).all()
    assert (host(gr.count) == og.count[::-1]).all()


def test_empty_input(ctx):
    e32 = torch.empty(0, dtype=torch.int32, device="cuda")
    e64 = torch.empty(0, dtype=torch.float64, device="cuda")
    gr = ctx.sort_groupby([e32], [e64], agg_cols=[0])
    assert gr.n_groups == 0


def _host_args(keys, payload, agg_cols, n, perm_in=None):
    """vdf_sort_groupby_args over numpy host arrays, with numpy output buffers."""
    import ctypes as C
    from visondf_b200 import _lib
    out = {"perm": np.empty(n, np.uint32), "gk": [np.empty(n, k.dtype) for k in keys], "cnt": np.empty(n, np.int64),
           "aggs": []}
    a = _lib.vdf_sort_groupby_args()
    kc = (_lib.vdf_col * len(keys))(*[_lib.vdf_col(k.ctypes.data, _lib_dt(k)) for k in keys])
    pc = (_lib.vdf_col * max(1, len(payload)))(*[_lib.vdf_col(p.ctypes.data, _lib_dt(p)) for p in payload])
    aggs = (_lib.vdf_agg_out * max(1, len(agg_cols)))()
    for i, c in enumerate(agg_cols):
        v = payload[c]
        f = v.dtype.kind == "f"
        o = {"sum": np.empty(n, np.float64 if f else np.int64), "hi": None if f else np.empty(n, np.int64),
             "min": np.empty(n, v.dtype), "max": np.empty(n, v.dtype), "mean": np.empty(n, np.float64)}
        out["aggs"].append(o)
        aggs[i] = _lib.vdf_agg_out(o["sum"].ctypes.data, None if f else o["hi"].ctypes.data, o["min"].ctypes.data,
                                   o["max"].ctypes.data, o["mean"].ctypes.data)
    gk = (C.c_void_p * len(keys))(*[g.ctypes.data for g in out["gk"]])
    ac = (C.c_int32 * max(1, len(agg_cols)))(*agg_cols)
    ng = C.c_uint64(0)
    a.n, a.keys, a.nkeys, a.order = n, kc, len(keys), 0
    a.payload, a.npayload = pc, len(payload)
    a.perm_out = out["perm"].ctypes.data
    a.groupby, a.agg_cols, a.nagg, a.aggs = 1, ac, len(agg_cols), aggs
    a.group_keys_out, a.group_count_out = gk, out["cnt"].ctypes.data
    a.n_groups_host = C.pointer(ng)
    if perm_in is not None:
        a.perm_in = perm_in.ctypes.data
    out["_keep"] = [kc, pc, aggs, gk, ac, keys, payload, perm_in]
    out["_ng"] = ng
    return a, out


def _lib_dt(a):
    from visondf_b200 import _lib
    return {np.dtype(np.int32): _lib.I32, np.dtype(np.int64): _lib.I64, np.dtype(np.uint32): _lib.U32,
            np.dtype(np.uint64): _lib.U64, np.dtype(np.float64): _lib.F64, np.dtype(np.float32): _lib.F32}[a.dtype]


def test_host_entry_point_matches_oracle(ctx):
    import ctypes as C
    rng = np.random.default_rng(41)
    keys, vals = frame(123_457, [np.int64, np.int32], 60, rng)
    a, out = _host_args(keys, vals, [0, 1], keys[0].size)
    st = vdf.lib.vdf_sort_groupby_host(ctx.handle, C.byref(a), None)
    assert st == 0, vdf.lib.vdf_ctx_last_error(ctx.handle)
    og = ob.groupby(keys, vals)
    g = int(out["_ng"].value)
    assert g == og.n_groups
    assert (out["perm"] == ob.argsort(keys)).all()
    for k, ok in zip(out["gk"], og.keys):
        assert (k[:g] == ok).all()
    assert (out["cnt"][:g] == og.count).all()
    assert (out["aggs"][1]["sum"][:g] == og.sum[1]).all() and (out["aggs"][1]["hi"][:g] == og.sum_hi[1]).all()
    assert (np.abs(out["aggs"][0]["sum"][:g] - og.sum[0]) <= 1e-12 * np.maximum(og.abs[0], 1e-300)).all()


def test_host_entry_point_with_input_permutation(ctx):
    # sorting through a row view composes the permutations (stable within the view)
    import ctypes as C
    rng = np.random.default_rng(42)
    n = 50_000
    k = rng.integers(0, 10, n).astype(np.int32)
    view = rng.permutation(n).astype(np.uint32)
    a, out = _host_args([k], [], [], n, perm_in=view)
    a.groupby = 0
    assert vdf.lib.vdf_sort_groupby_host(ctx.handle, C.byref(a), None) == 0
    exp = view[np.argsort(k[view], kind="stable")]
    assert (out["perm"] == exp).all()


def test_gather_host_and_transform_groupby_host(ctx):
    import ctypes as C
    from visondf_b200 import _lib
    rng = np.random.default_rng(43)
    n = 70_001
    perm = rng.permutation(n).astype(np.uint32)
    cols = [rng.standard_normal(n), rng.integers(-5, 5, n).astype(np.int32)]
    outs = [np.empty_like(c) for c in cols]
    ic = (_lib.vdf_col * 2)(*[_lib.vdf_col(c.ctypes.data, _lib_dt(c)) for c in cols])
    oc = (C.c_void_p * 2)(*[o.ctypes.data for o in outs])
    assert vdf.lib.vdf_gather_host(ctx.handle, n, perm.ctypes.data, ic, 2, oc, None) == 0
    for c, o in zip(cols, outs):
        assert bits_equal(o, c[perm])
    key = rng.integers(0, 300, n).astype(np.int64)
    val = rng.integers(-1000, 1000, n).astype(np.int32)
    og = ob.groupby([key], [val])
    lookup = {int(k): i for i, k in enumerate(og.keys[0])}
    gi = np.array([lookup[int(k)] for k in key])
    kc = (_lib.vdf_col * 1)(_lib.vdf_col(key.ctypes.data, _lib.I64))
    vc = _lib.vdf_col(val.ctypes.data, _lib.I32)
    ng = C.c_uint64(0)
    for fn, exp in [(0, og.count[gi]), (1, og.sum[0][gi]), (2, og.mean[0][gi]), (3, og.min[0][gi]), (4, og.max[0][gi])]:
        out = np.empty(n, np.int32 if fn in (3, 4) else (np.float64 if fn == 2 else np.int64))
        st = vdf.lib.vdf_transform_groupby_host(ctx.handle, n, kc, 1, vc, fn, None, out.ctypes.data, C.byref(ng), None)
        assert st == 0
        assert int(ng.value) == og.n_groups
        if fn == 2:
            np.testing.assert_allclose(out, exp, rtol=1e-12)
        else:
            assert (out == exp).all(), fn


@pytest.mark.parametrize("threshold", [1, 64, 200, 480, 512])
def test_striped_emit_threshold_gives_the_same_groups(threshold):
    """Every tile whose group starts reach the threshold takes the striped
    emit path (down to 1: groups of any length); the result is the oracle's
    either way."""
    c = vdf.Context(0)
    try:
        c.set_group_tuning(threshold)
        assert c.get_group_tuning() == threshold
        rng = np.random.default_rng(threshold)
        n = 300_001
        for pool in (n // 2, n // 4, 3000, 7):  # ~2, ~4, ~100, ~43,000 rows per group
            key = rng.integers(0, pool, n).astype(np.int64)
            v1 = rng.standard_normal(n)
            v2 = rng.integers(-10**12, 10**12, n)
            gr = c.sort_groupby([dev(key)], [dev(v1), dev(v2)], agg_cols=[0, 1])
            c.check()
            og = ob.groupby([key], [v1, v2])
            assert gr.n_groups == og.n_groups
            assert (host(gr.keys[0]) == og.keys[0]).all() and (host(gr.count) == og.count).all()
            a1, a2 = gr.aggs
            assert (host(a2.sum) == og.sum[1]).all() and (host(a2.sum_hi) == og.sum_hi[1]).all()
            assert (host(a2.min) == og.min[1]).all() and (host(a2.max) == og.max[1]).all()
            assert bits_equal(host(a1.min), og.min[0]) and bits_equal(host(a1.max), og.max[0])
            assert_f64_close(host(a1.sum), og.sum[0], og.abs[0], f"threshold {threshold} pool {pool} f64 sum")
        c.set_group_tuning(0)
        assert c.get_group_tuning() == 480
    finally:
        c.close()


# Tiles of the emit pass are 512 rows, four to a CTA of the two-value kernel;
# a tile range without a group head is skipped there, so boundaries at and
# beside those edges (and next to the last row) are the cases to pin.
EDGE_N = [2048 * 5, 2048 * 5 + 1, 2048 * 5 - 1, 2048 * 3 + 512, 1_000_003]


def edge_bounds(n, rng):
    cand = [1, 511, 512, 513, 1535, 2047, 2048, 2049, 4096, 4608, 6143, 200_000, 204_800, 204_801,
            n - 2049, n - 2048, n - 2047, n - 513, n - 512, n - 511, n - 2, n - 1]
    cand += list(rng.integers(1, n, 3))
    return sorted({int(b) for b in cand if 0 < b < n})


@pytest.mark.parametrize("n", EDGE_N)
@pytest.mark.parametrize("nvals", [2, 3])  # two values: the wide emit kernel; three: the per-tile one
@pytest.mark.parametrize("bounds", ["none", "last", "first", "edges"])
def test_few_groups_with_heads_at_tile_edges(ctx, n, nvals, bounds):
    rng = np.random.default_rng(n + nvals)
    b = {"none": [], "last": [n - 1], "first": [1], "edges": edge_bounds(n, rng)}[bounds]
    b = [x for x in b if 0 < x < n]
    key = np.zeros(n, np.int64)
    for x in b:
        key[x:] += 1
    key = key * 1_000_003 - 7  # sorted, distinct per group
    vals = [rng.standard_normal(n), rng.integers(-10**15, 10**15, n), rng.integers(-2**31, 2**31, n).astype(np.int32)]
    vals = vals[:nvals]
    og = ob.groupby([key], vals)
    for want_rg in (False, True):  # row_group wanted: every tile is emitted
        gr = ctx.groupby_sorted([dev(key)], [dev(v) for v in vals], want_row_group=want_rg, want_group_start=True)
        ctx.check()
        compare(og, gr, vals, f"n={n} bounds={bounds} row_group={want_rg}")
        assert (host(gr.group_start).view(np.uint32) == np.array([0] + b, np.uint32)).all()
        if want_rg:
            assert (host(gr.row_group).view(np.uint32) == (key + 7) // 1_000_003).all()
