"""The MSD-first radix sort (top-digit passes, chunks of whole buckets sorted
in shared memory, runs of equal high key bits ranked by the rest of the key)
against the CPU oracle, bit for bit, and its on-device fallback to the LSD
passes wherever the data defeats the plan.  A context with the MSD-first plan
forced at every size and key width makes small inputs take the same path as
the 100M-row ones."""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle_bind as ob
import visondf_b200 as vdf
from gpu_util import bits_equal, dev, host
from visondf_b200 import _lib, datagen

pytestmark = pytest.mark.gpu

ORDERS = [vdf.ORDER_ASC, vdf.ORDER_DESC_STABLE, vdf.ORDER_DESC_REVERSE]


@pytest.fixture(scope="module")
def mctx():
    c = vdf.Context(0)
    c.set_sort_strategy(_lib.SORT_MSD, 0)
    yield c
    c.close()


def run_sort(c, keys, order=vdf.ORDER_ASC):
    """Sorts through the C-ABI, checks against the oracle; returns (MSD sorts,
    fallbacks) this call added."""
    s0 = c.sort_stats()
    dk = [dev(k) for k in keys]
    sk = [torch.empty_like(k) for k in dk]
    perm = c.argsort(dk, order=order, sorted_keys_out=sk)
    c.check()
    s1 = c.sort_stats()
    exp = ob.argsort(keys, order)
    got = host(perm).view(np.uint32)
    assert got.shape == exp.shape
    bad = np.flatnonzero(got != exp)
    assert bad.size == 0, f"{bad.size} rows differ, first at {bad[0]}"
    for k, s in zip(keys, sk):
        assert bits_equal(host(s), k[exp])
    return s1["msd_sorts"] - s0["msd_sorts"], s1["msd_fallbacks"] - s0["msd_fallbacks"]


# chunks are 2048 nominal rows and at most 4096; one top digit up to 393,216
# rows, two above
SIZES = [2, 3, 31, 33, 2047, 2048, 2049, 4095, 4096, 4097, 100_003, 393_216, 393_217, 1_000_003]


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("dt", [np.int32, np.int64, np.uint32, np.uint64])
def test_uniform_integer_keys_take_the_msd_path(mctx, n, dt):
    rng = np.random.default_rng(n * 13 + np.dtype(dt).itemsize)
    keys = [datagen.keys_for("uniform", dt, n, rng)]
    used, fell = run_sort(mctx, keys)
    assert used == 1 and fell == 0


@pytest.mark.parametrize("n", [2, 4097, 100_003, 1_000_003])
@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_float_keys(mctx, n, dt):
    rng = np.random.default_rng(n + 5)
    run_sort(mctx, [datagen.keys_for("uniform", dt, n, rng)])


@pytest.mark.parametrize("dist", ["uniform", "few", "equal", "sorted", "reversed", "zipf", "small"])
@pytest.mark.parametrize("dt", [np.int32, np.int64, np.uint64, np.float64])
@pytest.mark.parametrize("order", ORDERS)
def test_distributions_and_orders(mctx, dist, dt, order):
    if dist in ("zipf", "small") and np.dtype(dt).kind == "f":
        pytest.skip("integer-only distribution")
    rng = np.random.default_rng(hash((dist, np.dtype(dt).name, order, 7)) & 0xFFFF)
    for n in (250_001, 700_001):
        run_sort(mctx, [datagen.keys_for(dist, dt, n, rng)], order)


def pool_keys(rng, n, pool, dtype):
    if np.dtype(dtype).kind == "f":
        values = rng.standard_normal(pool).astype(dtype)
    else:
        values = datagen.distinct_pool(rng, pool, dtype)
    return values[rng.integers(0, pool, size=n)]


@pytest.mark.parametrize("order", ORDERS)
@pytest.mark.parametrize("dts", [(np.int64, np.int32), (np.int32, np.int64), (np.float64, np.uint64),
                                 (np.uint32, np.uint32), (np.uint64, np.float32)])
@pytest.mark.parametrize("k0", ["uniform", "ties", "zipf"])
def test_two_keys(mctx, dts, k0, order):
    rng = np.random.default_rng(hash((k0, dts, order)) & 0xFFFF)
    n = 300_007
    if k0 == "ties":  # about two rows per primary value: ranked by key 1 in shared memory
        key0 = pool_keys(rng, n, n // 2, dts[0])
    else:
        key0 = datagen.keys_for(k0 if np.dtype(dts[0]).kind != "f" else "uniform", dts[0], n, rng)
    key1 = datagen.keys_for("zipf" if np.dtype(dts[1]).kind != "f" else "few", dts[1], n, rng)
    used, fell = run_sort(mctx, [key0, key1], order)
    assert used == 1
    if k0 in ("uniform", "ties") and np.dtype(dts[0]).kind != "f":
        assert fell == 0


def test_two_keys_ties_at_full_chunk_density(mctx):
    # the tie-heavy shape of the two-key workload at two top digits
    rng = np.random.default_rng(77)
    n = 1_500_001
    key0 = pool_keys(rng, n, n // 2, np.int64)
    key1 = datagen.keys_for("zipf", np.int32, n, rng)
    used, fell = run_sort(mctx, [key0, key1])
    assert (used, fell) == (1, 0)


def test_fallback_when_one_bucket_overflows_a_chunk(mctx):
    # passes the top-digit check, but one 16-bit bucket holds 50K rows
    rng = np.random.default_rng(1)
    k = datagen.keys_for("uniform", np.int64, 500_000, rng)
    k[rng.choice(500_000, 50_000, replace=False)] = k[0]
    used, fell = run_sort(mctx, [k])
    assert (used, fell) == (1, 1)


def test_long_unsorted_runs(mctx):
    # ~250 rows share each high 32-bit half, in random low-half order: a
    # one-key chunk finishes with more shared-memory passes ...
    rng = np.random.default_rng(2)
    n = 500_000
    hi = rng.integers(0, 1 << 32, 2000, dtype=np.uint64)[rng.integers(0, 2000, n)]
    k = (hi << np.uint64(32)) | rng.integers(0, 1 << 32, n, dtype=np.uint64)
    used, fell = run_sort(mctx, [k])
    assert (used, fell) == (1, 0)
    for order in ORDERS[1:]:
        assert run_sort(mctx, [k.view(np.int64)], order) == (1, 0)
    # ... and with a second key deciding (equal primaries, random key 1) the
    # plan falls back to the LSD passes
    k0 = pool_keys(rng, n, 2000, np.int64)
    k1 = datagen.keys_for("uniform", np.int32, n, rng)
    used, fell = run_sort(mctx, [k0, k1])
    assert (used, fell) == (1, 1)


def test_long_runs_of_equal_keys_need_no_fallback(mctx):
    # duplicates of one full key are already in row order
    rng = np.random.default_rng(3)
    k = pool_keys(rng, 500_000, 2000, np.int64)
    used, fell = run_sort(mctx, [k])
    assert (used, fell) == (1, 0)


def test_fallback_on_the_top_digit_check(mctx):
    used, fell = run_sort(mctx, [np.full(300_000, 7, np.int64)])
    assert (used, fell) == (1, 1)


def test_lsd_strategy_and_min_rows(ctx):
    c = vdf.Context(0)
    try:
        c.set_sort_strategy(_lib.SORT_LSD, 0)
        rng = np.random.default_rng(4)
        used, _ = run_sort(c, [datagen.keys_for("uniform", np.int64, 200_000, rng)])
        assert used == 0
        c.set_sort_strategy(_lib.SORT_AUTO, 300_000)
        used, _ = run_sort(c, [datagen.keys_for("uniform", np.int64, 200_000, rng)])
        assert used == 0
        used, _ = run_sort(c, [datagen.keys_for("uniform", np.int64, 300_000, rng)])
        assert used == 1
        assert c.get_sort_strategy() == (_lib.SORT_AUTO, 300_000)
        # the automatic choice leaves 4-byte key 0 to the LSD passes
        used, _ = run_sort(c, [datagen.keys_for("uniform", np.int32, 300_000, rng)])
        assert used == 0
        c.set_sort_strategy(_lib.SORT_MSD, 300_000)
        used, _ = run_sort(c, [datagen.keys_for("uniform", np.int32, 300_000, rng)])
        assert used == 1
        assert c.get_sort_strategy() == (_lib.SORT_MSD, 300_000)
    finally:
        c.close()


def test_sort_groupby_through_a_row_view(mctx):
    # the first top-digit pass reads the keys through the input permutation
    from test_groupby_gpu import _host_args
    rng = np.random.default_rng(5)
    n = 400_003
    k = datagen.keys_for("uniform", np.int64, n, rng)
    view = rng.permutation(n).astype(np.uint32)
    a, out = _host_args([k], [], [], n, perm_in=view)
    a.groupby = 0
    assert vdf.lib.vdf_sort_groupby_host(mctx.handle, C.byref(a), None) == 0
    exp = view[np.argsort(k[view], kind="stable")]
    assert (out["perm"] == exp).all()


def test_sort_groupby_two_keys_matches_oracle(mctx):
    rng = np.random.default_rng(6)
    n = 600_001
    keys = [pool_keys(rng, n, n // 3, np.int64), datagen.keys_for("zipf", np.int32, n, rng)]
    vals = [rng.standard_normal(n), rng.integers(-1000, 1000, n).astype(np.int32)]
    gr = mctx.sort_groupby([dev(k) for k in keys], [dev(v) for v in vals], agg_cols=[0, 1])
    mctx.check()
    perm = ob.argsort(keys)
    assert (host(gr.perm).view(np.uint32) == perm).all()
    og = ob.groupby(keys, vals)
    assert gr.n_groups == og.n_groups
    for g, o in zip(gr.keys, og.keys):
        assert (host(g) == o).all()
    assert (host(gr.count) == og.count).all()
    assert (host(gr.aggs[1].sum) == og.sum[1]).all()


@pytest.mark.parametrize("dt", [np.int32, np.int64, np.uint64])
@pytest.mark.parametrize("n,pool", [(300_000, 3), (300_000, 40), (300_000, 5000), (1_000_000, 2000),
                                    (1_000_000, 12_000)])
def test_long_runs_of_few_values_take_the_dense_bin_finish(mctx, dt, n, pool):
    # chunks where a bin holds more than 64 rows: stable passes over the
    # dense bin index (one for <= 256 occupied bins, two above), no fallback
    # unless a top-digit bucket overflows a chunk
    from test_batch_gpu import msd_plan_fails  # the chunk rules, emulated on the host
    rng = np.random.default_rng(pool * 7 + np.dtype(dt).itemsize)
    k = pool_keys(rng, n, pool, dt)
    used, fell = run_sort(mctx, [k])
    assert used == 1
    assert fell == int(msd_plan_fails(k, _lib.SORT_MSD))
    if pool >= 2000:
        assert fell == 0


def test_dense_bin_finish_with_mixed_runs(mctx):
    # long runs of one value next to spread keys in the same chunks (more
    # than 256 occupied bins), and bins holding two values of a long run
    rng = np.random.default_rng(8)
    n = 400_000
    k = datagen.keys_for("uniform", np.int64, n, rng)
    hot = datagen.distinct_pool(rng, 2000, np.int64)
    pick = rng.random(n) < 0.3
    k[pick] = hot[rng.integers(0, 2000, int(pick.sum()))]
    k[rng.random(n) < 0.01] += 1  # neighbours of hot values share their bins
    for order in ORDERS:
        used, fell = run_sort(mctx, [k], order)
        assert used == 1 and fell == 0


@pytest.mark.parametrize("dt", [np.int64, np.uint32, np.float64])
@pytest.mark.parametrize("dist", ["uniform", "ties", "few-long-runs"])
def test_wide_chunks(dt, dist):
    """Chunks of up to 8,192 rows (one CTA of 1024 threads) -- forced here at
    small sizes; planned by default where they save a top-digit pass."""
    c = vdf.Context(0)
    try:
        c.set_sort_strategy(_lib.SORT_MSD, 0)
        c.set_local_sort_variant(2)
        assert c.get_local_sort_variant() == 2
        rng = np.random.default_rng(hash((np.dtype(dt).name, dist)) & 0xFFFF)
        for n in (5000, 8193, 400_001, 2_000_003):
            if dist == "uniform":
                keys = [datagen.keys_for("uniform", dt, n, rng)]
            elif dist == "ties":
                keys = [pool_keys(rng, n, max(2, n // 2), dt), datagen.keys_for("zipf", np.int32, n, rng)]
            else:
                keys = [pool_keys(rng, n, max(2, n // 150), dt)]
            for order in ORDERS:
                used, fell = run_sort(c, keys, order)
                assert used == 1
                if dist == "uniform" and np.dtype(dt).kind != "f":
                    assert fell == 0
        c.set_local_sort_variant(3)  # with match.any
        run_sort(c, [datagen.keys_for("uniform", np.int64, 1_000_003, rng)])
    finally:
        c.close()
