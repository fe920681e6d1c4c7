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
