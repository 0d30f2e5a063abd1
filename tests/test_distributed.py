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


def _replica_energy_grads(specs):
    """Sum over `specs` of d(LJ pair energy)/d(eps, sigma) in FP64 (torch
    autograd over all minimum-image pairs within the cutoff, shifted as the
    replicas specify): a real per-replica gradient of shared parameters."""
    import numpy as np
    import torch

    eps = torch.tensor(np.asarray(specs[0].epsilon, np.float64), requires_grad=True)
    sig = torch.tensor(np.asarray(specs[0].sigma, np.float64), requires_grad=True)
    total = torch.zeros((), dtype=torch.float64)
    for s in specs:
        x = torch.tensor(np.asarray(s.positions, np.float64))
        box = torch.tensor(np.asarray(s.box_bound[1], np.float64) -
                           np.asarray(s.box_bound[0], np.float64))
        t = torch.tensor(np.asarray(s.types, np.int64) - 1)
        d = x[:, None, :] - x[None, :, :]
        d = d - box * torch.round(d / box)
        r2 = (d * d).sum(-1)
        iu = torch.triu_indices(len(x), len(x), 1)
        r2 = r2[iu[0], iu[1]]
        e = eps[t[iu[0]], t[iu[1]]]
        sg = sig[t[iu[0]], t[iu[1]]]
        keep = r2 < s.cutoff ** 2
        sr6 = (sg[keep] ** 2 / r2[keep]) ** 3
        shift = (sg[keep] ** 2 / s.cutoff ** 2) ** 3
        total = total + (4 * e[keep] * (sr6 * sr6 - sr6 - (shift * shift - shift))).sum()
    total.backward()
    return eps.grad.detach(), sig.grad.detach()


def _fit_specs():
    from beads_b200 import workloads

    return workloads.fit_mixture(n_replicas=5, n=216, seed=3)


def _grad_worker(rank: int, world: int, port: int, out) -> None:
    import datetime

    import torch.distributed as dist

    from beads_b200.distributed import reduce_gradients, shard_replicas

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    mine, specs = shard_replicas(_fit_specs(), world, rank)
    g_eps, g_sig = _replica_energy_grads(specs)
    reduce_gradients([g_eps, g_sig])
    out.put((rank, sorted(mine), g_eps.numpy(), g_sig.numpy()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_shared_gradients_to_the_single_rank_answer():
    import numpy as np

    specs = _fit_specs()
    want_eps, want_sig = _replica_energy_grads(specs)
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_grad_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted((q.get(timeout=180) for _ in range(world)), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shards = [r[1] for r in results]
    assert sorted(shards[0] + shards[1]) == list(range(len(specs)))
    assert shards[0] and shards[1]  # both ranks hold replicas
    for _, _, g_eps, g_sig in results:
        np.testing.assert_allclose(g_eps, want_eps.numpy(), rtol=1e-12, atol=0)
        np.testing.assert_allclose(g_sig, want_sig.numpy(), rtol=1e-12, atol=0)
