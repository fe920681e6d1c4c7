"""The dictionary plan of a one-key sort (at most 256 distinct keys: one
stable radix pass over each key's rank) against the CPU oracle, bit for
bit, in every order and for every key type, and its hand-over to the
MSD-first or LSD passes when the keys take more values (decided on the
device).  A context with the row threshold at 0 makes small inputs take the
same path as the 200M-row ones."""
import ctypes as C

import numpy as np
import pytest

import oracle_bind as ob
import visondf_b200 as vdf
from gpu_util import bits_equal, dev, host
from visondf_b200 import _lib, datagen

pytestmark = pytest.mark.gpu

ORDERS = [vdf.ORDER_ASC, vdf.ORDER_DESC_STABLE, vdf.ORDER_DESC_REVERSE]
DTYPES = [np.int32, np.int64, np.uint32, np.uint64, np.float64, np.float32]


@pytest.fixture(scope="module")
def dctx():
    c = vdf.Context(0)
    c.set_sort_strategy(_lib.SORT_AUTO, 0)
    yield c
    c.close()


def pool_of(rng, d, dt):
    if np.dtype(dt).kind == "f":
        base = np.array([-0.0, 0.0, np.inf, -np.inf, 1.5, -2.25], dtype=dt)
        vals = np.unique(np.concatenate([base, rng.standard_normal(max(0, d)).astype(dt)]))
        vals = vals[rng.permutation(vals.size)][:d]
        if d >= 2:  # both zeros: distinct order images
            vals[:2] = np.array([-0.0, 0.0], dtype=dt)
        return vals
    info = np.iinfo(dt)
    vals = datagen.distinct_pool(rng, d, dt)
    if d >= 3:  # the extremes: the all-ones order image among them
        vals[0], vals[1] = info.max, info.min
    return vals


def run_sort(c, key, order):
    s0 = c.sort_stats()
    dk = dev(key)
    sk = [dk.new_empty(dk.shape)]
    perm = c.argsort([dk], order=order, sorted_keys_out=sk)
    c.check()
    s1 = c.sort_stats()
    exp = ob.argsort([key], order)
    got = host(perm).view(np.uint32)
    bad = np.flatnonzero(got != exp)
    assert bad.size == 0, f"{bad.size} rows differ, first at {bad[0]}"
    assert bits_equal(host(sk[0]), key[exp])
    return s1["dict_sorts"] - s0["dict_sorts"], s1["dict_taken"] - s0["dict_taken"], s1


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("d", [1, 2, 16, 255, 256, 257, 5000])
def test_distinct_counts_and_types(dctx, dt, d):
    rng = np.random.default_rng(d * 7 + np.dtype(dt).itemsize)
    pool = pool_of(rng, d, dt)
    for n in (1, 3, 3071, 3073, 100_003):
        key = pool[rng.integers(0, pool.size, n)]
        tried, taken, _ = run_sort(dctx, key, vdf.ORDER_ASC)
        assert tried == (1 if n >= 2 else 0)  # one row needs no sort
        assert taken == (1 if n >= 2 and np.unique(key.view(f"u{key.itemsize}")).size <= 256 else 0)


@pytest.mark.parametrize("order", ORDERS)
@pytest.mark.parametrize("dt", [np.int32, np.uint64, np.float64])
def test_orders_at_size(dctx, order, dt):
    rng = np.random.default_rng(order + 11)
    pool = pool_of(rng, 16, dt)
    # skewed: most rows on two keys, like the 16-key group-by config
    p = np.full(16, 0.1 / 14)
    p[:2] = 0.45
    key = pool[rng.choice(16, 2_000_003, p=p)]
    tried, taken, _ = run_sort(dctx, key, order)
    assert (tried, taken) == (1, 1)


def test_hand_over_to_the_msd_and_lsd_plans(dctx):
    rng = np.random.default_rng(5)
    n = 1_000_003
    # 8-byte spread keys: dictionary overflow -> MSD-first (no fallback)
    k = datagen.keys_for("uniform", np.int64, n, rng)
    s0 = dctx.sort_stats()
    tried, taken, s1 = run_sort(dctx, k, vdf.ORDER_ASC)
    assert (tried, taken) == (1, 0)
    assert s1["msd_sorts"] - s0["msd_sorts"] == 1 and s1["msd_fallbacks"] == s0["msd_fallbacks"]
    # 4-byte keys with 300 values: dictionary overflow -> LSD passes
    k = pool_of(rng, 300, np.int32)[rng.integers(0, 300, n)]
    assert run_sort(dctx, k, vdf.ORDER_DESC_STABLE)[:2] == (1, 0)
    # 8-byte keys with 300 values of ~10,000 rows: overflow -> MSD-first, whose
    # buckets overflow a chunk -> LSD
    k = pool_of(rng, 300, np.uint64)[rng.integers(0, 300, 3 * n)]
    s0 = dctx.sort_stats()
    tried, taken, s1 = run_sort(dctx, k, vdf.ORDER_ASC)
    assert (tried, taken) == (1, 0)
    assert s1["msd_fallbacks"] - s0["msd_fallbacks"] == 1


def test_strategies_that_skip_it(ctx):
    rng = np.random.default_rng(6)
    key = pool_of(rng, 8, np.int32)[rng.integers(0, 8, 5_000_000)]
    for strat in (_lib.SORT_LSD, _lib.SORT_MSD):
        c = vdf.Context(0)
        try:
            c.set_sort_strategy(strat, 0)
            assert run_sort(c, key, vdf.ORDER_ASC)[:2] == (0, 0)
        finally:
            c.close()
    # the default context: 5M rows are above its row threshold (4 x 2^20)
    c = vdf.Context(0)
    try:
        assert run_sort(c, key, vdf.ORDER_ASC)[:2] == (1, 1)
        assert run_sort(c, key[:1000], vdf.ORDER_ASC)[:2] == (0, 0)
    finally:
        c.close()


def test_through_a_row_view_and_the_group_by(dctx):
    from test_groupby_gpu import _host_args
    rng = np.random.default_rng(7)
    n = 500_001
    key = pool_of(rng, 40, np.int64)[rng.integers(0, 40, n)]
    view = rng.permutation(n).astype(np.uint32)
    a, out = _host_args([key], [], [], n, perm_in=view)
    a.groupby = 0
    s0 = dctx.sort_stats()
    assert vdf.lib.vdf_sort_groupby_host(dctx.handle, C.byref(a), None) == 0
    assert dctx.sort_stats()["dict_taken"] - s0["dict_taken"] == 1
    assert (out["perm"] == view[np.argsort(key[view], kind="stable")]).all()
    # sort + gather + group-by of the 16-key shape
    k = pool_of(rng, 16, np.int32)[rng.integers(0, 16, 2_000_000)]
    v1 = np.exp(rng.standard_normal(k.size))
    v2 = rng.integers(0, 1 << 40, k.size)
    gr = dctx.sort_groupby([dev(k)], [dev(v1), dev(v2)], agg_cols=[0, 1])
    dctx.check()
    og = ob.groupby([k], [v1, v2])
    assert gr.n_groups == og.n_groups == 16
    assert (host(gr.keys[0]) == og.keys[0]).all() and (host(gr.count) == og.count).all()
    assert (host(gr.aggs[1].sum) == og.sum[1]).all()
    assert (np.abs(host(gr.aggs[0].sum) - og.sum[0]) <= 1e-12 * og.abs[0]).all()


def test_a_stalled_tile_of_the_dictionary_pass_is_reported():
    c = vdf.Context(0)
    try:
        c.set_sort_strategy(_lib.SORT_AUTO, 0)
        rng = np.random.default_rng(8)
        key = pool_of(rng, 12, np.int32)[rng.integers(0, 12, 1_000_000)]
        c.set_test_hooks(spin_limit=256, stall_tile=0)
        c.argsort([dev(key)])
        with pytest.raises(vdf.VdfError) as e:
            c.check()
        assert e.value.status == _lib.ERR_TIMEOUT
        c.set_test_hooks()
        assert run_sort(c, key, vdf.ORDER_ASC)[:2] == (1, 1)
    finally:
        c.close()
