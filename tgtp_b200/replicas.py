"""Host logic of the multi-GPU runs: one process per GPU, every rank scores its own independent
workload (sources and graphs are independent in tgtp, so there is no collective on the data
path), each rank times its own device, and the job's time is the slowest rank's.

Used by bench.py under torchrun (NCCL between GPUs) and tested with the gloo backend on CPU."""
from __future__ import annotations

import os


def rank_info():
    """(rank, world size, local rank) from the torchrun environment (1 process without it)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def workload_seed(base: int, rank: int) -> int:
    """Each replica's graph seed: weak scaling, per-rank work fixed as the world grows."""
    return base + rank


def slowest(values, device=None):
    """Element-wise maximum over all ranks of a list of floats (times); the input unchanged when
    the process group is not initialised or has one rank."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def job_rate(units_per_rank: float, slowest_seconds: float, world: int) -> float:
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    return world * units_per_rank / slowest_seconds
