"""Host logic of running independent replicas of the time step, one per GPU.

The path has no exchange step (one grid per GPU, no collectives on the data path), so
N ranks run N independent runs; the only cross-rank operations are the barrier around
the timed region and the max over ranks of the elapsed time.
"""
from __future__ import annotations

import os


def rank_info():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def replica_seed(base: int, rank: int) -> int:
    """Each replica starts from its own seeded perturbation."""
    return base + rank


def max_over_ranks(x: float, world: int, device=None) -> float:
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(points_per_step: int, steps: int, world: int, max_seconds: float) -> float:
    """Whole-job grid-point-steps per second: every rank advances its own run."""
    return points_per_step * steps * world / max_seconds
