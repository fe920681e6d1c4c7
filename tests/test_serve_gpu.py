"""The request loop on the GPU: a Poisson trace over a resident table, run
with continuous batching (two batches in flight), and every request's result
compared with the same request run alone through the single-query call
(vdf_sort_groupby): permutation, group keys, counts, integer sums and
min/max bit-exact; f64 sums and means within 1e-12 * sum|x|."""
import numpy as np
import pytest
import torch

import visondf_b200 as vdf
from gpu_util import bits_equal, host
from visondf_b200 import datagen, serve

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def table():
    f = datagen.frame_w0(n=2_000_000, distinct=10_000)
    return [torch.from_numpy(f[k]).cuda() for k in ("key", "v1", "v2")]


def make_trace(table, nreq, rate, median, seed, cap=1_000_000):
    key, v1, v2 = table
    rng = np.random.default_rng(seed)
    specs = datagen.stream_specs(nreq, rate, median_rows=median, cap_rows=cap, seed_col=seed)
    reqs = []
    for i, s in enumerate(specs):
        n = s["n"]
        o = int(rng.integers(0, key.numel() - n + 1))
        reqs.append(serve.Request(rid=i, arrival=s["t"], rows=n, key=key[o:o + n], vals=[v1[o:o + n], v2[o:o + n]],
                                  need_bytes=n * serve.out_bytes_per_row([True, False])))
    return reqs


def compare_with_alone(ctx, reqs):
    for r in reqs:
        b, q = r.result
        got = b.result(q)
        alone = ctx.sort_groupby([r.key], r.vals, agg_cols=[0, 1])
        assert (host(got.perm) == host(alone.perm)).all(), r.rid
        assert got.n_groups == alone.n_groups, r.rid
        assert bits_equal(host(got.keys), host(alone.keys[0])) and (host(got.count) == host(alone.count)).all()
        gf, gi = got.aggs
        af, ai = alone.aggs
        assert (host(gi.sum) == host(ai.sum)).all() and (host(gi.sum_hi) == host(ai.sum_hi)).all()
        assert bits_equal(host(gi.min), host(ai.min)) and bits_equal(host(gi.max), host(ai.max))
        assert bits_equal(host(gf.min), host(af.min)) and bits_equal(host(gf.max), host(af.max))
        g_rows = host(got.count)
        starts = np.concatenate([[0], np.cumsum(g_rows)[:-1]])
        vs = host(r.vals[0])[host(got.perm)]
        abs_sum = np.add.reduceat(np.abs(vs), starts) if len(starts) else np.zeros(0)
        assert np.all(np.abs(host(gf.sum) - host(af.sum)) <= 1e-12 * abs_sum + 1e-300)
        assert np.all(np.abs(host(gf.mean) - host(af.mean)) <= 1e-12 * abs_sum / g_rows + 1e-300)


def test_stream_results_equal_alone_results(ctx, table):
    ex = serve.BatchExecutor(0, slots=2, max_batch_rows=1 << 24)
    reqs = make_trace(table, nreq=60, rate=20_000.0, median=50_000, seed=1)
    loop = serve.Loop(ex, budget_bytes=40 * 10**9, fixed_bytes=ex.reserved_bytes, max_batch_rows=1 << 24)
    st = loop.run(reqs)
    assert st.requests == 60 and all(r.completed is not None for r in reqs)
    assert st.batches < 60  # requests were batched together
    compare_with_alone(ctx, reqs)


def test_graph_launched_batches_and_tight_budget(ctx, table):
    ex = serve.BatchExecutor(0, slots=2, max_batch_rows=1 << 22, use_graph=True)
    reqs = make_trace(table, nreq=40, rate=1e9, median=20_000, seed=2, cap=200_000)
    need = max(r.need_bytes for r in reqs)
    budget = ex.reserved_bytes + 3 * need  # about three requests in flight at a time
    loop = serve.Loop(ex, budget_bytes=budget, fixed_bytes=ex.reserved_bytes, max_batch_rows=1 << 22)
    st = loop.run(reqs)
    assert st.max_in_flight_bytes <= budget
    compare_with_alone(ctx, reqs)


def test_per_call_executor_serves_the_same_trace(ctx, table):
    ex = serve.PerCallExecutor(0)
    reqs = make_trace(table, nreq=20, rate=1e9, median=30_000, seed=3)
    loop = serve.Loop(ex, budget_bytes=40 * 10**9, max_batch_queries=1)
    st = loop.run(reqs)
    assert st.batches == 20
    for r in reqs:
        alone = ctx.sort_groupby([r.key], r.vals, agg_cols=[0, 1])
        assert (host(r.result.perm) == host(alone.perm)).all()
