"""The library's request loop (vdf_server_*) on the GPU: a Poisson trace of
requests over a resident table, each result compared with the same request
run alone (vdf_sort_groupby): permutation, group keys, counts, integer
aggregates bit-exact; f64 sums and means within 1e-12 * sum|x|.  Also the
budget bound, request states and refusals."""
import numpy as np
import pytest
import torch

import visondf_b200 as vdf
from gpu_util import bits_equal, host
from visondf_b200 import datagen, serve

pytestmark = pytest.mark.gpu

VDT = [torch.float64, torch.int64]


@pytest.fixture(scope="module")
def table():
    f = datagen.frame_w0(n=3_000_000, distinct=10_000)
    return [torch.from_numpy(f[k]).cuda() for k in ("key", "v1", "v2")]


def trace(table, nreq, rate, median, seed, cap=1_000_000):
    key, v1, v2 = table
    rng = np.random.default_rng(seed)
    out = []
    for i, s in enumerate(datagen.stream_specs(nreq, rate, median_rows=median, cap_rows=cap, seed_col=seed)):
        n = s["n"]
        o = int(rng.integers(0, key.numel() - n + 1))
        out.append(serve.Request(rid=i, arrival=s["t"], rows=n, key=key[o:o + n], vals=[v1[o:o + n], v2[o:o + n]]))
    return out


def same_as_alone(ctx, r, res):
    alone = ctx.sort_groupby([r.key], r.vals, agg_cols=[0, 1])
    assert (host(res.perm) == host(alone.perm)).all()
    assert res.n_groups == alone.n_groups
    assert bits_equal(host(res.keys), host(alone.keys[0])) and (host(res.count) == host(alone.count)).all()
    (gf, gi), (af, ai) = res.aggs, alone.aggs
    assert (host(gi.sum) == host(ai.sum)).all() and (host(gi.sum_hi) == host(ai.sum_hi)).all()
    assert bits_equal(host(gi.min), host(ai.min)) and bits_equal(host(gi.max), host(ai.max))
    assert bits_equal(host(gf.min), host(af.min)) and bits_equal(host(gf.max), host(af.max))
    cnt = host(res.count)
    starts = np.concatenate([[0], np.cumsum(cnt)[:-1]])
    absum = np.add.reduceat(np.abs(host(r.vals[0])[host(res.perm)]), starts)
    assert np.all(np.abs(host(gf.sum) - host(af.sum)) <= 1e-12 * absum + 1e-300)
    assert np.all(np.abs(host(gf.mean) - host(af.mean)) <= 1e-12 * absum / cnt + 1e-300)


@pytest.mark.parametrize("use_graph", [False, True])
def test_served_results_equal_alone_results(ctx, table, use_graph):
    srv = serve.Server(0, budget_bytes=60e9, slots=2, max_batch_rows=1 << 23, val_dtypes=VDT, use_graph=use_graph)
    reqs = trace(table, 80, rate=30_000.0, median=40_000, seed=11)
    st = serve.serve_trace(srv, reqs, keep_results=True)
    assert st.requests == 80 and st.batches < 80
    for r in reqs:
        same_as_alone(ctx, r, r.result)
        assert r.result.t_submit <= r.result.t_start <= r.result.t_done
    srv.close()


def test_budget_bounds_memory_in_flight(ctx, table):
    # the budget must cover the reserved workspaces: find them, then allow ~3 requests more
    probe = serve.Server(0, budget_bytes=60e9, slots=2, max_batch_rows=1 << 20, val_dtypes=VDT)
    fixed = probe.stats()["fixed_bytes"]
    probe.close()
    per_req = 200_000 * serve.out_bytes_per_row([True, False]) + 256
    srv = serve.Server(0, budget_bytes=fixed + 3 * per_req, slots=2, max_batch_rows=1 << 20, val_dtypes=VDT)
    reqs = trace(table, 30, rate=1e9, median=100_000, seed=12, cap=200_000)
    st = serve.serve_trace(srv, reqs, keep_results=False)
    s = srv.stats()
    assert s["max_in_use_bytes"] <= fixed + 3 * per_req
    # each batch holds at most 3 * per_req bytes of requests, whenever the
    # scheduler admitted it, so the batch count has a size-only lower bound
    need = sum(r.rows * serve.out_bytes_per_row([True, False]) + 256 for r in reqs)
    assert s["completed"] == 30 and st.batches >= -(-need // (3 * per_req)) and st.batches >= 2
    # a request that can never fit is refused at submission
    key, v1, v2 = table
    with pytest.raises(vdf.VdfError):
        srv.submit(key[:1_000_000], [v1[:1_000_000], v2[:1_000_000]])
    srv.close()


def test_request_states_and_release(ctx, table):
    key, v1, v2 = table
    srv = serve.Server(0, budget_bytes=60e9, slots=1, max_batch_rows=1 << 22, val_dtypes=VDT)
    ids = [srv.submit(key[i * 1000:(i + 1) * 1000 + i], [v1[i * 1000:(i + 1) * 1000 + i],
                                                       v2[i * 1000:(i + 1) * 1000 + i]]) for i in range(20)]
    # a slot takes its next batch once its previous batch's results are all
    # released, so results are checked and released one by one
    for i, rid in enumerate(ids):
        res = srv.wait(rid)
        state, again = srv.poll(rid)
        assert state == 2 and again.n_groups == res.n_groups
        assert res.perm.numel() == 1000 + i
        alone = ctx.sort_groupby([key[i * 1000:(i + 1) * 1000 + i]],
                                 [v1[i * 1000:(i + 1) * 1000 + i], v2[i * 1000:(i + 1) * 1000 + i]], agg_cols=[0, 1])
        assert (host(res.perm) == host(alone.perm)).all()
        srv.release(rid)
    with pytest.raises(vdf.VdfError):
        srv.release(ids[0])  # already released
    # empty request
    rid = srv.submit(key[:0], [v1[:0], v2[:0]])
    res = srv.wait(rid)
    assert res.n_groups == 0 and res.perm.numel() == 0
    srv.release(rid)
    srv.close()
