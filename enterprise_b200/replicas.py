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


def rank_chunks(n_src: int, world: int, rank: int, max_batch: int = 1024) -> list[tuple[int, int]]:
    """The chunks of a shared source list that rank `rank` of `world` runs.

    The list is cut as a replica set on one node cuts it (ent_replicas_plan:
    contiguous chunks of at most max_batch sources, at least one per rank
    while sources last); processes share no work counter, so chunk c goes to
    rank c % world."""
    from . import replicas_plan
    return [ch for c, ch in enumerate(replicas_plan(n_src, world, max_batch)) if c % world == rank]


def gather_rows(local: list, n_src: int, dist=None):
    """Assembles per-chunk results in input order on rank 0.

    local: [((begin, end), rows), ...] with rows a (end - begin) x V array for
    this rank's chunks. Returns the n_src x V array on rank 0 (and without a
    process group), None on the other ranks. One gather_object on every rank."""
    parts = local
    if dist is not None:
        got = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
        dist.gather_object(local, got, dst=0)
        if dist.get_rank() != 0:
            return None
        parts = [p for r in got for p in r]
    if not parts:
        return None
    V = parts[0][1].shape[1]
    out = np.empty((n_src, V), dtype=parts[0][1].dtype)
    seen = np.zeros(n_src, dtype=bool)
    for (b, e), rows in parts:
        if rows.shape != (e - b, V) or seen[b:e].any():
            raise ValueError(f"chunk ({b}, {e}) does not fit the plan")
        out[b:e] = rows
        seen[b:e] = True
    if not seen.all():
        raise ValueError("chunks do not cover every source")
    return out


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
