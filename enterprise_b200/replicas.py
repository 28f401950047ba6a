"""Replica bookkeeping for jobs on several GPUs of one node.

BFS sources and serving queries are independent, so a job on N GPUs is N
replicas: every rank (one process per GPU) holds its own copy of the graph,
takes its own seeded source set and traverses it with no collective on the
data path. The reference has no multi-GPU path (bfs_gpu_coalescing_mem takes
one gpu_id, bfs_gpu_opt.cuh:293-300). The only collectives are the barriers
around a timed region and the reductions below, which every rank calls in the
same order: the work done is summed over ranks and the time is the slowest
rank's, so a job's rate is (units all ranks processed) / (max rank time).

Works with any torch.distributed backend: pass the device the backend reduces
on ("cuda:<local rank>" for NCCL, "cpu" for gloo).
"""
from __future__ import annotations

import numpy as np

SOURCE_SEED_BASE = 0x50C0000


def source_seed(scale: int, rank: int = 0) -> int:
    """Seed of rank `rank`'s source set on a graph of the given scale."""
    return SOURCE_SEED_BASE + scale + 1000 * rank


def rank_sources(beg_pos: np.ndarray, scale: int, rank: int, count: int) -> np.ndarray:
    """Seeded non-isolated sources of one rank (distinct within the rank)."""
    from . import pick_sources
    return pick_sources(beg_pos, source_seed(scale, rank), count)


def _reduce(x: float, dist, device, op_name: str) -> float:
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def max_over_ranks(x: float, dist=None, device="cpu") -> float:
    """Maximum of x over all ranks (x itself without a process group)."""
    return _reduce(x, dist, device, "MAX")


def sum_over_ranks(x: float, dist=None, device="cpu") -> float:
    """Sum of x over all ranks (x itself without a process group)."""
    return _reduce(x, dist, device, "SUM")


def job_rate(local_units: float, local_seconds: float, dist=None, device="cpu"):
    """(total units, job seconds, units per second) of a replicated job.

    Two collectives, SUM then MAX, in that order on every rank."""
    units = sum_over_ranks(local_units, dist, device)
    secs = max_over_ranks(local_seconds, dist, device)
    if secs <= 0:
        raise ValueError("job time must be positive")
    return units, secs, units / secs
