"""Multi-rank bookkeeping of `bench.py --gpus N` on CPU: two gloo ranks with
different step times agree on the slowest one, and the whole-job rate counts
every rank's rows over it.  The reference arm prints only on rank 0."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, results):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    from visondf_b200 import replicas

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        m = replicas.max_over_ranks(ms, world, "cpu")
        results[rank] = (m, replicas.whole_job_rate(1_000_000, world, m))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        results = mgr.dict()
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, results)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        got = dict(results)
    assert got[0] == got[1]
    m, rate = got[0]
    assert m == 15.0
    assert rate == pytest.approx(2 * 1_000_000 / 0.015)


def test_single_rank_is_identity():
    sys.path.insert(0, str(ROOT))
    from visondf_b200 import replicas

    assert replicas.max_over_ranks(3.5, 1) == 3.5
    assert replicas.whole_job_rate(100, 1, 1000.0) == 100.0


def test_reference_arm_prints_only_on_rank_zero():
    sys.path.insert(0, str(ROOT))
    import bench

    class A:
        steps, warmup, ref_sample = 1, 0, 1000

    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.reference_arm(A(), rank=1, world=2)
    assert buf.getvalue() == ""


def test_reference_arm_line_on_rank_zero():
    import json

    sys.path.insert(0, str(ROOT))
    import bench

    class A:
        steps, warmup, ref_sample = 1, 0, 20_000

    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.reference_arm(A(), rank=0, world=1)
    line = json.loads(buf.getvalue())
    assert line["impl"] == "reference" and line["unit"] == "rows/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
