"""Replica sharding and the rank bookkeeping of the multi-GPU path, on CPU with
two gloo ranks (the path itself has no data collective)."""

from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

from beads_b200.distributed import shard_by_atoms


def test_shards_cover_every_replica_once_and_balance_atoms():
    sizes = [256, 32768, 4000, 4100, 9000, 300, 12000, 700]
    shards = shard_by_atoms(sizes, 3)
    flat = sorted(r for s in shards for r in s)
    assert flat == list(range(len(sizes)))
    loads = [sum(sizes[r] for r in s) for s in shards]
    assert max(loads) - min(loads) <= max(sizes)
    assert shard_by_atoms(sizes, 3) == shards  # deterministic
    assert shard_by_atoms(sizes, 1) == [list(range(len(sizes)))]
    with pytest.raises(ValueError):
        shard_by_atoms(sizes, 0)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out) -> None:
    import datetime

    import torch.distributed as dist

    from beads_b200.distributed import gather_to_rank0, max_over_ranks, sum_over_ranks

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    sizes = [1000, 2000, 3000, 4000, 5000]
    mine = shard_by_atoms(sizes, world)[rank]
    atoms = sum(sizes[r] for r in mine)
    slowest = max_over_ranks(1.0 + rank)
    total = sum_over_ranks(atoms)
    gathered = gather_to_rank0([(rank, r) for r in mine], world)
    out.put((rank, slowest, total, gathered))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_time_and_work():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slowest, total, gathered in results:
        assert slowest == 2.0  # max over ranks of 1 + rank
        assert total == 15000.0  # every replica counted once
        if rank == 0:
            assert sorted(r for _, r in gathered) == [0, 1, 2, 3, 4]
        else:
            assert gathered is None
