"""The seeded workload generators (CPU): the polymer melt's two growth
orders keep the same invariants (no two beads closer than the rejection
radius, every bond of the step length, chains of the asked size) and are
reproducible from the seed; ``relaxed`` hands the descent a roomy list and
carries its positions and images back (engine stood in by a fake)."""

from __future__ import annotations

import numpy as np
import pytest
from scipy.spatial import cKDTree

from beads_b200 import workloads


def _check_melt(spec, n_chains, beads, reject=0.8, step=0.97):
    length = float(spec.box_bound[1][0])
    pos = np.asarray(spec.positions, np.float64)
    assert pos.shape == (n_chains * beads, 3)
    assert (pos >= 0.0).all() and (pos < length).all()
    tree = cKDTree(np.mod(pos, length), boxsize=length)
    # float32 storage moves a coordinate by at most ~length * 6e-8
    assert not tree.query_pairs(reject - 1e-5)
    chain = pos.reshape(n_chains, beads, 3)
    d = np.diff(chain, axis=1)
    d -= length * np.round(d / length)
    bond = np.linalg.norm(d, axis=2)
    assert np.allclose(bond, step, atol=2e-5)
    assert len(spec.bonds) == n_chains * (beads - 1)
    assert len(spec.angles) == n_chains * (beads - 2)
    assert len(spec.dihedrals) == n_chains * (beads - 3)


@pytest.mark.parametrize("growth", ["sequential", "lockstep"])
def test_polymer_melt_invariants(growth):
    spec = workloads.polymer_melt(n_chains=30, beads=40, seed=11, growth=growth)
    _check_melt(spec, 30, 40)


def test_lockstep_melt_is_seeded():
    a = workloads.polymer_melt(n_chains=50, beads=60, seed=4, growth="lockstep")
    b = workloads.polymer_melt(n_chains=50, beads=60, seed=4, growth="lockstep")
    c = workloads.polymer_melt(n_chains=50, beads=60, seed=5, growth="lockstep")
    assert np.array_equal(a.positions, b.positions)
    assert not np.array_equal(a.positions, c.positions)
    _check_melt(a, 50, 60)


def test_lockstep_melt_crowded_small_box():
    # A box of 2 grid cells per axis (the 27-cell stencil wraps onto itself)
    # and one of 4 coarse cells per axis (cells wider than 2 / sqrt(3) of
    # the rejection radius, so more than 8 beads may share one).
    for n_chains, beads in ((2, 5), (4, 12)):
        spec = workloads.polymer_melt(n_chains=n_chains, beads=beads, density=0.85, seed=2,
                                      growth="lockstep")
        _check_melt(spec, n_chains, beads)


def test_unknown_growth_refused():
    with pytest.raises(ValueError, match="unknown growth"):
        workloads.polymer_melt(n_chains=2, beads=4, growth="spiral")


def test_relaxed_carries_positions_images_and_capacity(monkeypatch):
    # Engine stand-in (the descent itself runs on the GPU): records the list
    # capacity it was built with and returns moved, partly wrapped positions.
    import beads_b200.engine as engine_mod

    seen = {}

    class FakeEngine:
        def __init__(self, spec):
            seen["capacity"] = spec.max_neighbors
            self.n = spec.n
            self.hi = float(spec.box_bound[1][0])

        def __enter__(self):
            return self

        def __exit__(self, *exc):
            return False

        def minimize(self, iterations, dmax, fref):
            seen["args"] = (iterations, dmax, fref)

        def state(self):
            pos = np.full((self.n, 3), 0.5, np.float32)
            pos[0, 0] = self.hi  # a coordinate that rounded onto the upper bound
            img = np.zeros((self.n, 3), np.int32)
            img[1] = (1, 0, -1)
            return {"positions": pos, "images": img}

    monkeypatch.setattr(engine_mod, "Engine", FakeEngine)
    spec = workloads.polymer_melt(n_chains=3, beads=6, seed=1, max_neighbors=64)
    out = workloads.relaxed(spec, iterations=7, dmax=0.02, fref=50.0)
    assert seen == {"capacity": 256, "args": (7, 0.02, 50.0)}
    assert out.max_neighbors == 64 and spec.max_neighbors == 64
    assert out.positions.dtype == np.float32
    assert (out.positions < np.float32(spec.box_bound[1][0])).all()
    assert tuple(out.images[1]) == (1, 0, -1)
    assert np.array_equal(out.bonds, spec.bonds)
    assert out is not spec and not np.array_equal(out.positions, spec.positions)
