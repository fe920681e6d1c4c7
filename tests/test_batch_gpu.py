"""Batched queries (vdf_batch_*): every query of a mixed batch against the
oracle, the same batch under every tuning (one-CTA path, segmented path,
4/8/11-bit digits, tile sizes), graph replay, and each query alone versus in
the mix.  Bit-exact for permutations, group keys, counts, integer sums and
min/max; f64 sums and means within 1e-12 * sum|x| (f64 sums may differ in
the last bits between a query run alone and in a mix, since the segmented
reduction's tiles fall differently)."""
import numpy as np
import pytest
import torch

import oracle_bind as ob
import visondf_b200 as vdf
from gpu_util import assert_f64_close, bits_equal, dev, host
from visondf_b200 import _lib, datagen

pytestmark = pytest.mark.gpu

KEY_TYPES = [np.int32, np.int64, np.uint32, np.uint64, np.float64, np.float32]


def make_queries(specs):
    out = []
    for i, (n, dt, card) in enumerate(specs):
        rng = np.random.default_rng(9000 + i)
        if np.dtype(dt).kind == "f":
            pool = rng.standard_normal(max(1, card)).astype(dt)
            if card > 3:
                pool[:3] = np.array([-0.0, np.inf, -np.inf], dtype=dt)
        else:
            pool = datagen.distinct_pool(rng, max(1, card), dt)
        key = pool[rng.integers(0, len(pool), size=n)] if n else np.empty(0, dt)
        v1 = rng.standard_normal(n)
        v2 = rng.integers(-10**15, 10**15, size=n, dtype=np.int64)
        out.append((key, v1, v2))
    return out


SPECS = [(0, np.int32, 1), (1, np.int64, 1), (7, np.uint32, 3), (1000, np.int32, 10), (4096, np.int64, 2048),
         (4097, np.int32, 4), (8192, np.float64, 100), (2048, np.float32, 50), (20_000, np.uint64, 5000),
         (150_001, np.int64, 40_000), (33_333, np.int32, 2), (70_000, np.float64, 1000), (3, np.int64, 3),
         (500, np.uint64, 1), (90_000, np.int32, 45_000), (6000, np.uint32, 6000)]


def to_batch(ctx, queries, tuning=None):
    qs = [(dev(k), [dev(v1), dev(v2)]) for k, v1, v2 in queries]
    return vdf.Batch(ctx, qs, tuning), qs


def check_against_oracle(b, queries):
    for q, (key, v1, v2) in enumerate(queries):
        r = b.result(q)
        n = key.size
        if n == 0:
            assert r.n_groups == 0 and r.perm.numel() == 0
            continue
        assert (host(r.perm).view(np.uint32) == ob.argsort([key])).all(), q
        og = ob.groupby([key], [v1, v2])
        assert r.n_groups == og.n_groups, q
        assert bits_equal(host(r.keys), og.keys[0]), q
        assert (host(r.count) == og.count).all(), q
        a1, a2 = r.aggs
        assert (host(a2.sum) == og.sum[1]).all() and (host(a2.sum_hi) == og.sum_hi[1]).all(), q
        assert bits_equal(host(a2.min), og.min[1]) and bits_equal(host(a2.max), og.max[1]), q
        assert bits_equal(host(a1.min), og.min[0]) and bits_equal(host(a1.max), og.max[0]), q
        assert_f64_close(host(a1.sum), og.sum[0], og.abs[0], f"query {q} f64 sum")
        assert_f64_close(host(a1.mean), og.mean[0], og.abs[0] / og.count, f"query {q} f64 mean")
        assert_f64_close(host(a2.mean), og.mean[1], np.abs(og.mean[1]), f"query {q} int mean")


def snapshot(b, nq):
    out = []
    for q in range(nq):
        r = b.result(q)
        out.append([host(r.perm), r.n_groups, host(r.keys), host(r.count)] +
                   [host(x) for a in r.aggs for x in (a.sum, a.sum_hi, a.min, a.max, a.mean) if x is not None])
    return out


def test_mixed_batch_matches_the_oracle(ctx):
    queries = make_queries(SPECS)
    b, _ = to_batch(ctx, queries)
    info = b.info()
    assert info["small_queries"] > 0 and info["large_queries"] > 0
    b.launch()
    ctx.check()
    check_against_oracle(b, queries)
    b.close()


@pytest.mark.parametrize("seg_variant", range(len(_lib.batch_variants())))
@pytest.mark.parametrize("small", [(0, 8), (4096, 4), (8192, 8), (8192, 4)])
def test_every_tuning_matches_the_oracle(ctx, seg_variant, small):
    queries = make_queries(SPECS)
    b, _ = to_batch(ctx, queries, dict(small_rows=small[0], small_bits=small[1], seg_variant=seg_variant))
    b.launch()
    ctx.check()
    check_against_oracle(b, queries)
    b.close()


SPECS_4BYTE_LARGE = [(3, np.int64, 3), (1000, np.uint64, 10), (70_000, np.int32, 1000), (150_001, np.float32, 40_000),
                     (20_000, np.uint32, 20_000), (33_333, np.int32, 2), (5000, np.float64, 700)]


@pytest.mark.parametrize("seg_variant", range(len(_lib.batch_variants())))
def test_four_byte_key_arena_matches_the_oracle(ctx, seg_variant):
    """Every large query has 4-byte keys, so the arena holds 4-byte key
    images; small queries of 8-byte keys run on the one-CTA path beside it."""
    queries = make_queries(SPECS_4BYTE_LARGE)
    b, _ = to_batch(ctx, queries, dict(small_rows=8192, small_bits=8, seg_variant=seg_variant))
    assert b.info()["large_queries"] == 4
    b.launch()
    ctx.check()
    check_against_oracle(b, queries)
    b.close()


def test_graph_replay_gives_the_same_bits(ctx):
    queries = make_queries(SPECS)
    b, _ = to_batch(ctx, queries)
    b.launch()
    ctx.check()
    ref = snapshot(b, len(queries))
    for _ in range(3):
        b.perm.fill_(-1)
        b.count.fill_(-1)
        b.launch_graph()
        ctx.check()
        got = snapshot(b, len(queries))
        for x, y in zip(ref, got):
            assert all(bits_equal(np.asarray(u), np.asarray(v)) for u, v in zip(x, y))
    b.close()


def test_each_query_alone_equals_the_mix(ctx):
    queries = make_queries(SPECS)
    b, _ = to_batch(ctx, queries)
    b.launch()
    ctx.check()
    mixed = snapshot(b, len(queries))
    for q, one in enumerate(queries):
        a, _ = to_batch(ctx, [one])
        a.launch()
        ctx.check()
        alone = snapshot(a, 1)[0]
        m = mixed[q]
        assert (alone[0] == m[0]).all() and alone[1] == m[1]
        assert bits_equal(alone[2], m[2]) and (alone[3] == m[3]).all()
        # f64 sum / mean: within tolerance; everything else bit-identical
        f_sum, f_min, f_max, f_mean = alone[4:8]
        assert bits_equal(f_min, m[5]) and bits_equal(f_max, m[6])
        absum = np.abs(one[1]).sum() if one[1].size else 0.0
        assert np.all(np.abs(f_sum - m[4]) <= 1e-12 * absum + 1e-300)
        for u, v in zip(alone[8:], m[8:]):
            if u.dtype == np.float64:
                assert np.all(np.abs(u - v) <= 1e-12 * np.abs(v) + 1e-300)
            else:
                assert bits_equal(u, v)
        a.close()
    b.close()


def test_generated_batch_shape_and_parity_sample(ctx):
    """A scaled-down batch from the batched-workload generator (400 queries,
    same distributions), every query checked."""
    specs = datagen.batch_specs(nq=400, budget_bytes=64 << 20, min_rows=1000, seed_col=1)
    queries = [datagen.batch_query(s) for s in specs]
    b, _ = to_batch(ctx, queries)
    b.launch_graph()
    ctx.check()
    check_against_oracle(b, queries)
    b.close()


def test_edge_batches(ctx):
    # all queries empty
    b, _ = to_batch(ctx, make_queries([(0, np.int32, 1), (0, np.int64, 1)]))
    b.launch()
    ctx.check()
    assert b.result(0).n_groups == 0 and b.result(1).n_groups == 0
    b.close()
    # one row; all rows one key; a single query of exactly the one-CTA limit
    for spec in [(1, np.float64, 1), (50_000, np.int64, 1), (8192, np.int32, 8192)]:
        queries = make_queries([spec])
        for small in (0, 8192):
            b, _ = to_batch(ctx, queries, dict(small_rows=small, small_bits=8, seg_variant=0))
            b.launch()
            ctx.check()
            check_against_oracle(b, queries)
            b.close()


def test_batch_rejects_bad_tuning_and_arguments(ctx):
    queries = make_queries([(10, np.int32, 3)])
    with pytest.raises(vdf.VdfError):
        to_batch(ctx, queries, dict(small_rows=10_000, small_bits=8, seg_variant=0))
    with pytest.raises(vdf.VdfError):
        to_batch(ctx, queries, dict(small_rows=0, small_bits=6, seg_variant=0))
    with pytest.raises(vdf.VdfError):
        to_batch(ctx, queries, dict(small_rows=0, small_bits=8, seg_variant=99))
    k = dev(queries[0][0])
    with pytest.raises(ValueError):
        vdf.Batch(ctx, [(k, [dev(queries[0][1]), dev(queries[0][2].astype(np.float64))]),
                        (k, [dev(queries[0][1]), dev(queries[0][2])])])


@pytest.mark.parametrize("vals", [(), (np.float32,), (np.int32, np.uint64, np.float64),
                                  (np.uint32, np.int64, np.float32, np.float64)])
def test_value_column_sets(ctx, vals):
    """No values, one value column (column gather), three and four columns
    (32-byte records with zero-padded slots), every value dtype."""
    rng = np.random.default_rng(4242 + len(vals))
    specs = [(3000, np.int64, 40), (50_000, np.int32, 900), (0, np.int32, 1), (120_000, np.uint64, 7),
             (7000, np.float64, 7000)]
    queries = []
    for n, kdt, card in specs:
        pool = datagen.distinct_pool(rng, card, kdt) if np.dtype(kdt).kind != "f" else rng.standard_normal(card)
        key = pool[rng.integers(0, card, size=n)].astype(kdt) if n else np.empty(0, kdt)
        vs = []
        for vdt in vals:
            if np.dtype(vdt).kind == "f":
                vs.append(rng.standard_normal(n).astype(vdt))
            else:
                info = np.iinfo(vdt)
                lo, hi = max(info.min, -10**12), min(info.max, 10**12)
                vs.append(rng.integers(lo, hi, size=n, dtype=vdt, endpoint=True))
        queries.append((key, vs))
    for small in (0, 4096):
        b = vdf.Batch(ctx, [(dev(k), [dev(v) for v in vs]) for k, vs in queries],
                      dict(small_rows=small, small_bits=8, seg_variant=0))
        b.launch()
        ctx.check()
        for q, (key, vs) in enumerate(queries):
            r = b.result(q)
            if key.size == 0:
                assert r.n_groups == 0
                continue
            assert (host(r.perm).view(np.uint32) == ob.argsort([key])).all()
            og = ob.groupby([key], vs) if vs else ob.groupby([key], [np.zeros(key.size)])
            assert r.n_groups == og.n_groups and bits_equal(host(r.keys), og.keys[0])
            assert (host(r.count) == og.count).all()
            for j, v in enumerate(vs):
                a = r.aggs[j]
                assert bits_equal(host(a.min), og.min[j]) and bits_equal(host(a.max), og.max[j]), (q, j)
                if v.dtype.kind == "f":
                    assert_f64_close(host(a.sum), og.sum[j], og.abs[j], f"query {q} col {j}")
                else:
                    assert (host(a.sum) == og.sum[j]).all() and (host(a.sum_hi) == og.sum_hi[j]).all(), (q, j)
        b.close()


# queries of the MSD-first plan: spread keys (one and two top digits, 8- and
# 4-byte), few distinct values (a bucket larger than a chunk: that query falls
# back to the LSD passes), one key for all rows (likewise), 8-byte keys whose
# high halves repeat (long runs finished by shared-memory passes)
SPECS_MSD = [(300_000, np.int64, 300_000), (4097, np.int32, 4097), (50_000, np.int64, 3), (393_217, np.uint32, 10**6),
             (9000, np.float64, 9000), (60_000, np.int32, 1), (2000, np.int64, 5), (120_000, np.uint64, 60_000),
             (25_000, np.float32, 25_000)]


def msd_queries():
    queries = make_queries(SPECS_MSD)
    rng = np.random.default_rng(41)
    n = 100_000
    hi = rng.integers(0, 1 << 31, 1000, dtype=np.int64)[rng.integers(0, 1000, n)]
    k = (hi << 32) | rng.integers(0, 1 << 32, n, dtype=np.int64)
    queries.append((k, rng.standard_normal(n), rng.integers(-10**15, 10**15, size=n, dtype=np.int64)))
    return queries


def order_image(key):
    """Unsigned image whose order is the key's (ints: sign bit flipped;
    floats: sign-magnitude to two's order)."""
    w = key.itemsize
    u = key.view(np.uint64 if w == 8 else np.uint32).astype(np.uint64)
    top = np.uint64(1 << (8 * w - 1))
    if key.dtype.kind == "i":
        return u ^ top
    if key.dtype.kind == "f":
        full = np.uint64((1 << (8 * w)) - 1)
        return np.where(u & top, ~u & full, u | top)
    return u


def msd_top_passes(key, strategy=_lib.SORT_AUTO):
    """Top-digit passes of a large query's MSD-first plan in a batch (0: the
    LSD passes): the fewest that leave about 1536 rows per bucket, at most
    three and fewer than the key's digits; 4-byte keys only when the MSD
    strategy is forced."""
    n, w = key.size, key.itemsize
    passes = [p for p in range(1, min(3, w - 1) + 1) if n <= 1536 << (8 * p)]
    if not passes or (w == 4 and strategy != _lib.SORT_MSD):
        return 0
    return passes[0]


def msd_plan_fails(key, strategy=_lib.SORT_AUTO):
    """Whether the MSD-first plan of one large query falls back to the LSD
    passes: chunks start every 2048 rows, moved forward to the next change of
    the top-digit bucket if one lies within 4096 rows, and no chunk may hold
    more than 4096 rows."""
    n, w = key.size, key.itemsize
    p = msd_top_passes(key, strategy)
    if not p:
        return False
    b = np.sort(order_image(key) >> np.uint64(8 * (w - p)))
    starts = [0]
    for x in range(2048, n, 2048):
        i = int(np.searchsorted(b, b[x - 1], side="right"))
        if i <= min(x + 4095, n - 1):
            starts.append(i)
        else:
            if x + 4095 < n - 1:
                return True
            starts.append(n)
    starts.append(n)
    return any(e - s > 4096 for s, e in zip(starts, starts[1:]))


@pytest.mark.parametrize("strategy", [_lib.SORT_AUTO, _lib.SORT_MSD])
@pytest.mark.parametrize("seg_variant", [0, 4])
def test_msd_plan_with_per_query_fallback_matches_lsd_plan(ctx, seg_variant, strategy):
    queries = msd_queries()
    tuning = dict(small_rows=4096, small_bits=8, seg_variant=seg_variant)
    m = vdf.Context(0)
    l = vdf.Context(0)
    try:
        m.set_sort_strategy(strategy, 0)
        l.set_sort_strategy(_lib.SORT_LSD, 0)
        bm, _ = to_batch(m, queries, tuning)
        bl, _ = to_batch(l, queries, tuning)
        large = bm.info()["large_queries"]
        msd = sum(msd_top_passes(k, strategy) > 0 for k, _, _ in queries if k.size > 4096)
        assert 0 < msd and (msd < large) == (strategy == _lib.SORT_AUTO)  # 4-byte queries: LSD under AUTO
        assert bm.sort_info() == dict(msd_queries=msd, lsd_queries=large - msd)
        assert bl.sort_info() == dict(msd_queries=0, lsd_queries=large)
        bm.launch()
        m.check()
        # the three-value and the one-value queries defeat the plan, and the
        # normal floats (most share a top byte); the others do not
        fails = [msd_plan_fails(k, strategy) for k, _, _ in queries if k.size > 4096]
        assert fails[2] and not fails[0] and not fails[-1]
        assert bm.sort_info(fallbacks=True)["fallbacks"] == sum(fails)
        check_against_oracle(bm, queries)
        bl.launch()
        l.check()
        ref = snapshot(bl, len(queries))
        for rep in range(2):  # replays re-arm the per-query flags
            bm.perm.fill_(-1)
            bm.launch_graph() if rep else bm.launch()
            m.check()
            got = snapshot(bm, len(queries))
            for q, (x, y) in enumerate(zip(ref, got)):
                assert (x[0] == y[0]).all() and x[1] == y[1], q
                assert bits_equal(x[2], y[2]) and (x[3] == y[3]).all(), q
        bm.close()
        bl.close()
    finally:
        m.close()
        l.close()


def test_four_byte_arena_takes_the_msd_plan_when_forced(ctx):
    queries = make_queries(SPECS_4BYTE_LARGE)
    tuning = dict(small_rows=8192, small_bits=8, seg_variant=4)
    auto, _ = to_batch(ctx, queries, tuning)
    assert auto.sort_info()["msd_queries"] == 0  # AUTO: 4-byte keys take the LSD passes
    auto.close()
    m = vdf.Context(0)
    try:
        m.set_sort_strategy(_lib.SORT_MSD, 0)
        b, _ = to_batch(m, queries, tuning)
        assert b.sort_info()["msd_queries"] == 4
        b.launch()
        m.check()
        fails = sum(msd_plan_fails(k, _lib.SORT_MSD) for k, _, _ in queries if k.size > 8192)
        assert fails >= 1  # the two-value query at least
        assert b.sort_info(fallbacks=True)["fallbacks"] == fails
        check_against_oracle(b, queries)
        b.close()
    finally:
        m.close()
