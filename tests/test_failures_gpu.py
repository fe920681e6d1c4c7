"""Failure paths that really trigger, none of them faulting the device: a
look-back wait that runs out (one tile of the first radix pass never
publishes its counts, and the poll limit is short), an injected workspace
allocation failure, and server batches that fail when they start or when
their results are read back.  After each, the same context or server serves
the next call correctly."""
import numpy as np
import pytest
import torch

import oracle_bind as ob
import visondf_b200 as vdf
from gpu_util import dev, host
from visondf_b200 import _lib, datagen, serve

pytestmark = pytest.mark.gpu


def sorts_correctly(c, k):
    perm = c.argsort([dev(k)])
    c.check()
    assert (host(perm).view(np.uint32) == ob.argsort([k])).all()


def _bulk64():
    return [v["index"] for v in _lib.sort_variants() if v["tma"] and v["key_width"] == 8][0]


@pytest.mark.parametrize("strategy,bulk", [(_lib.SORT_LSD, False), (_lib.SORT_AUTO, False), (_lib.SORT_LSD, True)])
def test_lookback_wait_runs_out_and_is_reported(strategy, bulk):
    c = vdf.Context(0)
    try:
        c.set_sort_strategy(strategy, 0)
        if bulk:  # the persistent bulk-load variant: the stalled tile's CTA goes on to later tiles
            c.set_sort_tuning(c.get_sort_tuning()[0], _bulk64())
        rng = np.random.default_rng(1)
        k = datagen.keys_for("uniform", np.int64, 2_000_000, rng)
        c.set_test_hooks(spin_limit=256, stall_tile=0)
        c.argsort([dev(k)])
        with pytest.raises(vdf.VdfError) as e:
            c.check()
        assert e.value.status == _lib.ERR_TIMEOUT
        c.check()  # the error bits were read and cleared
        c.set_test_hooks()
        sorts_correctly(c, k)
    finally:
        c.close()


def test_workspace_allocation_failure_leaves_the_context_usable():
    c = vdf.Context(0)
    try:
        rng = np.random.default_rng(2)
        k = datagen.keys_for("uniform", np.int32, 300_000, rng)
        v = rng.standard_normal(300_000)
        c.set_test_hooks(fail_allocs=1)
        with pytest.raises(vdf.VdfError) as e:
            c.sort_groupby([dev(k)], [dev(v)], agg_cols=[0])
        assert e.value.status == _lib.ERR_OOM
        sorts_correctly(c, k)  # the hook is used up: this call allocates
        gr = c.sort_groupby([dev(k)], [dev(v)], agg_cols=[0])
        assert gr.n_groups == ob.groupby([k], [v]).n_groups
    finally:
        c.close()


@pytest.mark.parametrize("where", ["start", "finish"])
def test_server_batch_failure_surfaces_and_later_requests_are_served(where):
    rng = np.random.default_rng(3)
    n = 50_000
    key = dev(rng.integers(0, 100, n).astype(np.int32))
    v1 = dev(rng.standard_normal(n))
    v2 = dev(rng.integers(-10**6, 10**6, n))
    srv = serve.Server(0, budget_bytes=4e9, slots=2, max_batch_rows=1 << 20, val_dtypes=[torch.float64, torch.int64])
    try:
        srv.inject_failure(where, 1, _lib.ERR_DEVICE)
        rid = srv.submit(key, [v1, v2])
        with pytest.raises(vdf.VdfError) as e:
            srv.wait(rid)
        assert e.value.status == _lib.ERR_DEVICE
        with pytest.raises(vdf.VdfError):  # polling a failed request reports its status too
            srv.poll(rid)
        srv.release(rid)
        og = ob.groupby([host(key)], [host(v1), host(v2)])
        for _ in range(2):
            rid = srv.submit(key, [v1, v2])
            r = srv.wait(rid)
            assert r.n_groups == og.n_groups
            assert (host(r.count) == og.count).all()
            assert (host(r.aggs[1].sum) == og.sum[1]).all()
            srv.release(rid)
        st = srv.stats()
        assert st["in_use_bytes"] == st["fixed_bytes"]  # every request's memory came back
    finally:
        srv.close()
