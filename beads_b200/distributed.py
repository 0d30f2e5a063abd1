"""Replica sharding across GPUs (one process per GPU).

The path has no exchange step: replicas are independent, so a batch is split
across ranks by atom count and every rank runs its share in one batched
engine.  The only collectives are bookkeeping: a barrier around the timed
region, the maximum of the per-rank times, and gathering per-replica results
on rank 0 (NCCL on GPUs, gloo in the CPU tests).
"""

from __future__ import annotations

import heapq
from typing import Sequence


def shard_by_atoms(sizes: Sequence[int], world: int) -> list[list[int]]:
    """Greedy longest-processing-time split of replica indices over `world`
    ranks by particle count; deterministic for a given `sizes`."""
    if world < 1:
        raise ValueError("world size must be positive")
    order = sorted(range(len(sizes)), key=lambda r: (-int(sizes[r]), r))
    heap = [(0, rank) for rank in range(world)]
    heapq.heapify(heap)
    shards: list[list[int]] = [[] for _ in range(world)]
    for r in order:
        load, rank = heapq.heappop(heap)
        shards[rank].append(r)
        heapq.heappush(heap, (load + int(sizes[r]), rank))
    return [sorted(s) for s in shards]


def max_over_ranks(value: float, device=None) -> float:
    """Largest `value` over all ranks (the time of the slowest rank)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_to_rank0(items: list, world: int) -> list | None:
    """Concatenated per-rank lists on rank 0 (None elsewhere)."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return list(items)
    out = [None] * world if dist.get_rank() == 0 else None
    dist.gather_object(items, out, dst=0)
    if out is None:
        return None
    return [x for part in out for x in part]
