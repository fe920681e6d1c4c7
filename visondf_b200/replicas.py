"""Replica bookkeeping for multi-GPU runs.

The sort + group-by path does not shard: `bench.py --gpus N` runs N
independent replicas, one process per GPU.  Each rank times its own steps on
the device; the job's time is the slowest rank's (an all-reduce MAX over the
process group) and the job's throughput is every rank's rows over that time.
"""
from __future__ import annotations


def max_over_ranks(value: float, world: int, device=None) -> float:
    """The maximum of `value` over all ranks (identity when world == 1).
    `device` is where the reduction tensor lives: a CUDA device for NCCL, the
    CPU for gloo."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: int, world: int, ms_max: float) -> float:
    """Units per second of the whole job: all ranks' units over the slowest
    rank's time per step (weak scaling: per-rank work is fixed)."""
    return units_per_rank * world / (ms_max / 1e3)
