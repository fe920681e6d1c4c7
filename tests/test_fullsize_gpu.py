"""Full-size runs of the workload shapes, checked through properties that do
not need the CPU oracle (too slow at these sizes) and through an independent
recomputation with torch on the same GPU:

  * the permutation is a permutation of [0, n) and orders the keys
    lexicographically, stably (ties keep row order);
  * sorted keys and gathered payloads equal the inputs indexed by it;
  * group keys strictly increase and equal the first row of their group,
    counts equal torch.bincount over the row groups and sum to n, min/max
    equal torch.scatter_reduce, integer sums are exact to the last bit of the
    128-bit result (recomputed from 20-bit halves on a sample of groups), f64
    sums are within 1e-12 * sum|x| of an independent sum.

The 1M-row frame is compared with the oracle directly.
"""
import numpy as np
import pytest
import torch

import oracle_bind as ob
from gpu_util import bits_equal, dev, host
from visondf_b200 import datagen

pytestmark = pytest.mark.gpu

F64_REL = 1e-12


@pytest.fixture(autouse=True)
def _release_cache():
    yield
    torch.cuda.empty_cache()


def check_permutation(perm, n):
    p = perm.view(torch.int32).long()
    assert int(p.min()) == 0 and int(p.max()) == n - 1
    seen = torch.zeros(n, dtype=torch.int8, device=p.device)
    seen[p] = 1
    assert int(seen.sum()) == n


def lex_lt_eq(cols):
    """(a[i] < a[i+1], a[i] == a[i+1]) lexicographically over the columns."""
    lt = torch.zeros(cols[0].numel() - 1, dtype=torch.bool, device=cols[0].device)
    eq = torch.ones_like(lt)
    for k in cols:
        a, b = k[:-1], k[1:]
        lt |= eq & (a < b)
        eq &= a == b
    return lt, eq


def check_sorted_stable(sorted_keys, perm):
    lt, eq = lex_lt_eq(sorted_keys)
    p = perm.view(torch.int32)
    ok = lt | (eq & (p[:-1] < p[1:]))
    assert bool(ok.all()), f"order broken at {int((~ok).nonzero()[0])}"


def reference_f64_sums(v, rg, g, gs, cnt):
    """Per-group sums and sums of |x| of f64 values sorted by group.  Few
    large groups: numpy's pairwise sum over each contiguous slice on the
    host; many small groups: index_add on the device (a handful of
    additions per group)."""
    if g <= 64:
        vh = host(v)
        starts, counts = host(gs).astype(np.int64), host(cnt)
        s = np.array([vh[a:a + c].sum() for a, c in zip(starts, counts)])
        sa = np.array([np.abs(vh[a:a + c]).sum() for a, c in zip(starts, counts)])
        return torch.from_numpy(s).to(v.device), torch.from_numpy(sa).to(v.device)
    s = torch.zeros(g, dtype=torch.float64, device=v.device).index_add_(0, rg, v)
    sa = torch.zeros(g, dtype=torch.float64, device=v.device).index_add_(0, rg, v.abs())
    return s, sa


def check_int_sums(v, rg, g, agg, sample=200_000):
    """The library's 128-bit sum (hi * 2^64 + unsigned lo) against an exact
    recomputation: sum(x) = 2^20 * sum(x >> 20) + sum(x & (2^20 - 1)), both
    partial sums far inside int64."""
    x = v.long()
    s_lo = torch.zeros(g, dtype=torch.int64, device=x.device).scatter_add_(0, rg, x & ((1 << 20) - 1))
    s_hi = torch.zeros(g, dtype=torch.int64, device=x.device).scatter_add_(0, rg, x >> 20)
    if g <= sample:  # every group
        idx = np.arange(g)
    else:
        rng = np.random.default_rng(0)
        idx = np.unique(np.concatenate([rng.integers(0, g, size=sample), [0, g - 1]]))
    it = torch.from_numpy(idx).to(x.device)
    got = [int(h) * (1 << 64) + int(l) for h, l in
           zip(host(agg.sum_hi[it]), host(agg.sum[it]).view(np.uint64))]
    want = [int(h) * (1 << 20) + int(l) for h, l in zip(host(s_hi[it]), host(s_lo[it]))]
    assert got == want


def check_groups(gr, sorted_vals, n):
    g = gr.n_groups
    rg = gr.row_group.view(torch.int32).long()
    assert int(rg[0]) == 0 and int(rg[-1]) == g - 1
    cnt = torch.bincount(rg, minlength=g)
    assert torch.equal(cnt, gr.count) and int(gr.count.sum()) == n
    gs = gr.group_start.view(torch.int32).long()
    assert torch.equal(gs[1:], torch.cumsum(cnt, 0)[:-1])
    for k_sorted, k_group in zip(gr.sorted_keys, gr.keys):
        assert torch.equal(k_sorted[gs], k_group)
    if g > 1:
        lt, _ = lex_lt_eq(gr.keys)
        assert bool(lt.all())
    for v, a in zip(sorted_vals, gr.aggs):
        if v.dtype == torch.float64:
            mn = torch.full((g,), float("inf"), dtype=v.dtype, device=v.device).scatter_reduce_(0, rg, v, "amin")
            mx = torch.full((g,), float("-inf"), dtype=v.dtype, device=v.device).scatter_reduce_(0, rg, v, "amax")
            assert torch.equal(mn, a.min) and torch.equal(mx, a.max)
            s, sa = reference_f64_sums(v, rg, g, gs, cnt)
            err = (a.sum - s).abs()
            assert bool((err <= F64_REL * sa + 1e-300).all())
            plain = int((err > F64_REL * s.abs()).sum())
            print(f"f64 sums: {g} groups within 1e-12 * sum|x|; plain-relative failures: {plain}")
            mean = a.sum / gr.count.double()
            assert bool(((a.mean - mean).abs() <= F64_REL * mean.abs() + 1e-300).all())
        else:
            x = v.long()
            big, small = torch.iinfo(torch.int64).max, torch.iinfo(torch.int64).min
            mn = torch.full((g,), big, dtype=torch.int64, device=v.device).scatter_reduce_(0, rg, x, "amin")
            mx = torch.full((g,), small, dtype=torch.int64, device=v.device).scatter_reduce_(0, rg, x, "amax")
            assert torch.equal(mn, a.min.long()) and torch.equal(mx, a.max.long())
            check_int_sums(v, rg, g, a)


def signed(t):
    """Unsigned tensors viewed as signed ones of the same width (indexing and
    comparisons of uint64 are not implemented for every torch op)."""
    return t.view({torch.uint32: torch.int32, torch.uint64: torch.int64}.get(t.dtype, t.dtype))


def run_full(ctx, keys_h, pay_h, agg_cols):
    keys = [dev(k) for k in keys_h]
    pay = [dev(p) for p in pay_h]
    gr = ctx.sort_groupby(keys, pay, agg_cols=agg_cols, want_row_group=True, want_group_start=True)
    ctx.check()
    n = keys[0].numel()
    check_permutation(gr.perm, n)
    check_sorted_stable(gr.sorted_keys, gr.perm)
    p = gr.perm.view(torch.int32).long()
    for k, s in zip(keys, gr.sorted_keys):
        assert torch.equal(signed(k)[p], signed(s))
    for v, s in zip(pay, gr.payload):
        assert torch.equal(signed(v)[p], signed(s))
    del p, keys, pay
    check_groups(gr, [gr.payload[c] for c in agg_cols], n)
    return gr


def test_one_million_rows_against_the_oracle(ctx):
    f = datagen.frame_w0()
    keys, vals = [f["key"]], [f["v1"], f["v2"]]
    gr = ctx.sort_groupby([dev(k) for k in keys], [dev(v) for v in vals], agg_cols=[0, 1])
    ctx.check()
    assert (host(gr.perm).view(np.uint32) == ob.argsort(keys)).all()
    og = ob.groupby(keys, vals)
    assert gr.n_groups == og.n_groups == 10_000
    assert bits_equal(host(gr.keys[0]), og.keys[0]) and (host(gr.count) == og.count).all()
    a_f, a_i = gr.aggs
    assert (host(a_i.sum) == og.sum[1]).all() and (host(a_i.sum_hi) == og.sum_hi[1]).all()
    assert bits_equal(host(a_i.min), og.min[1]) and bits_equal(host(a_i.max), og.max[1])
    assert bits_equal(host(a_f.min), og.min[0]) and bits_equal(host(a_f.max), og.max[0])
    assert (np.abs(host(a_f.sum) - og.sum[0]) <= F64_REL * og.abs[0]).all()


def test_hundred_million_rows_two_keys(ctx):
    f = datagen.frame_w1()
    gr = run_full(ctx, [f["key1"], f["key2"]], [f["f64"], f["i32"], f["rowid"]], [0, 1])
    assert gr.n_groups > 99_000_000
    # the row-id payload is the permutation itself
    assert torch.equal(gr.payload[2].view(torch.int64), gr.perm.view(torch.int32).long())


def test_two_hundred_million_rows_fifty_million_keys(ctx):
    f = datagen.frame_w2a()
    gr = run_full(ctx, [f["key"]], [f["v1"], f["v2"]], [0, 1])
    assert 48_500_000 < gr.n_groups <= 50_000_000


def test_two_hundred_million_rows_sixteen_skewed_keys(ctx):
    f = datagen.frame_w2b()
    gr = run_full(ctx, [f["key"]], [f["v1"], f["v2"]], [0, 1])
    assert gr.n_groups == 16
    assert int(gr.count.max()) > 89_000_000
    # sums of 2^40-range values over ~90M rows pass 2^64: the high word is used
    assert int(gr.aggs[1].sum_hi.max()) > 0
