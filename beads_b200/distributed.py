"""Replica sharding across GPUs (one process per GPU).

The MD path has no exchange step: replicas are independent, so a batch is
split across ranks by atom count and every rank runs its share in one batched
engine.  The one data collective is the differentiable fit's: parameters
shared by all replicas get the sum of every rank's gradient (one FP64
all-reduce per backward pass).  The rest is bookkeeping: a barrier around the
timed region, the maximum of the per-rank times, and gathering per-replica
results on rank 0 (NCCL on GPUs, gloo in the CPU tests).
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


def shard_replicas(specs: Sequence, world: int, rank: int) -> tuple[list[int], list]:
    """This rank's replicas of one batch description: (indices, specs),
    split by shard_by_atoms over the replicas' particle counts.  Every rank
    builds the same description, so no data moves between ranks."""
    mine = shard_by_atoms([int(s.n) for s in specs], world)[rank]
    return mine, [specs[r] for r in mine]


def reduce_gradients(tensors, device=None) -> None:
    """Sums, in place, gradients of parameters shared by the replicas of every
    rank (LJ and bonded tables, the loss): each rank holds the sum over its
    own replicas, the all-reduce gives every rank the whole batch's sum (NCCL
    on GPUs, gloo on CPU).  FP64, one collective for all tensors, in the
    order given (the same order on every rank).  A no-op without an
    initialised process group."""
    import torch
    import torch.distributed as dist

    tensors = [t for t in tensors if t is not None]
    if not tensors or not (dist.is_available() and dist.is_initialized()):
        return
    flat = torch.cat([t.detach().reshape(-1).to(torch.float64) for t in tensors])
    if device is not None:
        flat = flat.to(device)
    dist.all_reduce(flat, op=dist.ReduceOp.SUM)
    flat = flat.cpu()
    at = 0
    for t in tensors:
        k = t.numel()
        t.copy_(flat[at:at + k].reshape(t.shape).to(t.dtype))
        at += k
