"""Cell-tile staging of the pair forces against the slot layout, on the GPU.

A staged context keeps its list rows in cell order with stage indices as
entries and reads every neighbour position of the pair loop from a
shared-memory copy of the group's stencil cells (k_lj_staged); the slot
layout gathers them from global memory (k_lj).  Same arithmetic, same list
order, same canonical summation order: the two must give the same bits --
forces at step 0, energies and virial, and the whole state after a run with
rebuilds, reorders and thermostat.  Covered: the binary mixture (sorted at
every rebuild), the LJ lattice, a bead-spring melt (exclusions and bonded
terms), a batch of uneven replicas (staged and unstaged replicas side by
side), the fit mixture (sorted every 10th rebuild, so staging gathers through
the cell order), and a slab of crowded cells whose groups overflow the stage
capacity and fall back to slot entries inside a staged context.
"""

from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from beads_b200 import workloads
from beads_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _mixture():
    spec = workloads.lj_mixture(n=12000, box=(12000 / 20.37) ** (1 / 3), seed=11,
                                max_neighbors=160)
    with Engine(spec) as eng:
        eng.minimize(300, 0.004, 200.0)
        spec.positions = workloads._inside(eng.state()["positions"].astype(np.float64),
                                           np.zeros(3), np.asarray(spec.box_bound[1], float))
    return [spec]


def _slab():
    """Dense slab (x < L/4) in a sparse box: groups in the slab exceed the
    stage capacity sized for the mean occupancy."""
    rng = np.random.default_rng(8)
    box = 12.0
    dense = rng.uniform(0.0, 1.0, (9000, 3)) * [box / 4, box, box]
    sparse = rng.uniform(0.0, 1.0, (3000, 3)) * [3 * box / 4, box, box] + [box / 4, 0, 0]
    spec = workloads.lj_lattice()
    pos = np.concatenate([dense, sparse])
    spec.positions = workloads._inside(pos, np.zeros(3), np.full(3, box))
    n = pos.shape[0]
    spec.types = np.ones(n, np.int32)
    spec.velocities = np.zeros((n, 3), np.float32)
    spec.masses = np.ones(n, np.float32)
    spec.box_bound = np.array([[0, 0, 0], [box] * 3], np.float32)
    spec.sigma = np.array([[0.2]])
    spec.cutoff, spec.cutoff_buffer = 1.0, 0.2
    spec.max_neighbors = 1024
    return [spec]


CASES = {
    "mixture": _mixture,
    "lattice": lambda: [workloads.lj_lattice()],
    "melt": lambda: [workloads.polymer_melt(n_chains=40, beads=50, seed=3, max_neighbors=96)],
    "batch": lambda: workloads.replica_batch(6, n_min=256, n_max=8000, seed=4),
    "fit": lambda: workloads.fit_mixture(n_replicas=2, n=8192),
}


def _run(specs, staged: bool, steps: int):
    with Engine(specs) as eng:
        eng.set_list_staged(staged)
        obs0 = eng.eval()
        st0 = [eng.state(r) for r in range(len(specs))]
        obs1 = eng.run(steps, steps) if steps else None
        st1 = [eng.state(r) for r in range(len(specs))] if steps else None
        layout = eng.list_staged()
        counts = [eng.debug_neighbors(r) for r in range(len(specs))]
    return layout, obs0, st0, obs1, st1, counts


@pytest.mark.parametrize("which", list(CASES))
def test_staged_layout_gives_the_slot_layout_bits(which):
    specs = CASES[which]()
    a = _run(specs, True, 200)
    b = _run(specs, False, 200)
    assert a[0] is True and b[0] is False  # the staged context really staged
    for key in ("pair_pe", "bond_pe", "angle_pe", "dihedral_pe", "virial"):
        for r in range(len(specs)):
            assert a[1][r][key] == b[1][r][key], (which, r, key)
            assert a[3][r][key] == b[3][r][key], (which, r, key)
    for r in range(len(specs)):
        assert np.array_equal(a[2][r]["forces"], b[2][r]["forces"]), (which, r)
        for key in ("positions", "velocities", "forces", "images"):
            assert np.array_equal(a[4][r][key], b[4][r][key]), (which, r, key)
        # the decoded staged list is the same list, entry for entry
        assert np.array_equal(a[5][r][0], b[5][r][0])
        assert np.array_equal(a[5][r][1], b[5][r][1])


def test_groups_beyond_the_stage_capacity_fall_back_inside_a_staged_context():
    specs = _slab()
    a = _run(specs, True, 0)
    b = _run(specs, False, 0)
    assert a[0] is True
    assert np.array_equal(a[2][0]["forces"], b[2][0]["forces"])
    assert a[1][0]["pair_pe"] == b[1][0]["pair_pe"]
    assert np.array_equal(a[5][0][0], b[5][0][0])
    assert np.array_equal(a[5][0][1], b[5][0][1])


def test_adjoint_leaves_the_staged_layout():
    import torch

    from beads_b200.adjoint import trajectory_observables

    specs = workloads.fit_mixture(n_replicas=1, n=2048)
    with Engine(specs) as eng:
        assert eng.list_staged()
        eps = torch.tensor(specs[0].epsilon, dtype=torch.float64, requires_grad=True)
        sig = torch.tensor(specs[0].sigma, dtype=torch.float64, requires_grad=True)
        x = torch.tensor(specs[0].positions, dtype=torch.float64, requires_grad=True)
        v = torch.tensor(specs[0].velocities, dtype=torch.float64)
        obs = trajectory_observables(eng, eps, sig, x, v, steps=10, record_from=1,
                                     checkpoint_every=5)
        obs[:, :, 0].sum().backward()
        assert not eng.list_staged()
        assert torch.isfinite(eps.grad).all() and torch.isfinite(x.grad).all()
    # a replica of the same input with the slot layout from the start agrees
    spec2 = dataclasses.replace(specs[0])
    with Engine([spec2]) as eng2:
        eng2.set_list_staged(False)
        eps2 = eps.detach().clone().requires_grad_(True)
        sig2 = sig.detach().clone().requires_grad_(True)
        x2 = torch.tensor(specs[0].positions, dtype=torch.float64, requires_grad=True)
        obs2 = trajectory_observables(eng2, eps2, sig2, x2, v, steps=10, record_from=1,
                                      checkpoint_every=5)
        obs2[:, :, 0].sum().backward()
    assert torch.equal(obs, obs2)
    assert torch.equal(eps.grad, eps2.grad) and torch.equal(x.grad, x2.grad)
