"""Replica (data-parallel) bookkeeping for runs of one process per GPU.

Horn-Schunck pairs are independent, so N GPUs run N replicas with no collective on the data
path: rank r processes its own pair (seeded base + r), and the whole job's rate is all
ranks' work divided by the slowest rank's time.  The only collective is the max over ranks
of the measured times (NCCL on GPUs; gloo works the same on CPU).
"""
from __future__ import annotations

from typing import List, Optional, Sequence


def rank_seed(base: int, rank: int) -> int:
    """Seed of rank `rank`'s synthetic pair."""
    return base + rank


def max_over_ranks(values: Sequence[float], group=None, device: Optional[str] = None) -> List[float]:
    """Element-wise max of `values` over all ranks of the default process group (the
    values unchanged when no group is initialised).  `device` is where the reduction
    buffer lives: "cuda" for NCCL, "cpu" for gloo (default: by backend)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return [float(v) for v in values]
    if device is None:
        device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return t.tolist()


def job_rate(units_per_rank: float, world: int, seconds: float) -> float:
    """Whole-job throughput: every rank's units over the slowest rank's seconds."""
    return units_per_rank * world / seconds
