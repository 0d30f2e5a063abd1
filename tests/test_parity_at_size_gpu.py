"""The CUDA engine against the FP64 oracle at the benchmark configurations'
own sizes, through the C ABI.

  * the 1,048,576-bead binary mixture in its 37.2 nm box, relaxed as the
    benchmark relaxes it (the box where the exactly rounded minimum image
    decides whether boundary pairs stay inside the force bar), at step 0 and
    after 100 MD steps;
  * a 50,000-bead bead-spring melt grown and relaxed like the 400,000-bead
    one (pairs with 1-2/1-3 exclusions, bonds, angles, dihedrals);
  * the first 32 replicas of the 512-replica batch generator plus a
    256-bead replica (2 cells per axis), stepped as one batch;
  * two replicas of the 64 x 8192-bead fit mixture.

Bars: forces relative RMS <= 1e-5 against FP64; pair energy and virial
within 1e-5 relative (bonded energies likewise).
"""

from __future__ import annotations

import numpy as np
import pytest

from beads_b200 import workloads
from beads_b200.engine import Engine
from tests.helpers import oracle_forces, rel_rms

pytestmark = pytest.mark.gpu

FORCE_TOL = 1.0e-5
ENERGY_TOL = 1.0e-5


def _check(spec, obs, forces, positions=None):
    f64, e64, w64 = oracle_forces(spec, positions)
    err = rel_rms(forces, f64)
    assert err <= FORCE_TOL, f"force rel RMS {err:.3e}"
    floor = 1e-6 * spec.n
    for key, want in (("pair_pe", e64[0]), ("bond_pe", e64[1]), ("angle_pe", e64[2]),
                      ("dihedral_pe", e64[3]), ("virial", w64)):
        got = obs[key]
        assert abs(got - want) <= max(ENERGY_TOL * abs(want), floor), (key, got, want)
    return err


def test_mixture_1m_vs_fp64():
    spec = workloads.relaxed(workloads.lj_mixture(), iterations=500, dmax=0.004, fref=200.0,
                             capacity=256)
    assert spec.n == 1_048_576
    with Engine(spec) as eng:
        obs = eng.eval()[0]
        st = eng.state()
        _check(spec, obs, st["forces"])
        # 100 MD steps later: the list is the one of the last rebuild, the
        # oracle's is fresh; both must give the same forces.
        eng.run(99)
        obs = eng.run(1, 1)[0]
        st = eng.state()
    _check(spec, obs, st["forces"], positions=st["positions"])


def test_melt_50k_vs_fp64():
    spec = workloads.relaxed(workloads.polymer_melt(n_chains=250, beads=200, seed=5,
                                                    growth="lockstep"))
    with Engine(spec) as eng:
        obs = eng.eval()[0]
        st = eng.state()
    _check(spec, obs, st["forces"])
    assert obs["bond_pe"] > 0 and obs["angle_pe"] > 0 and obs["dihedral_pe"] > 0


def test_replica_batch_slice_vs_fp64():
    specs = workloads.replica_batch(32) + workloads.replica_batch(1, n_min=256, n_max=256,
                                                                   seed=99)
    assert specs[-1].n == 256
    with Engine(specs) as eng:
        obs = eng.eval()
        states = [eng.state(r) for r in range(len(specs))]
        paths = {eng.debug_plan(r)["path"] for r in range(len(specs))}
    assert "direct" in paths or "small_dimension" in paths
    for r, spec in enumerate(specs):
        _check(spec, obs[r], states[r]["forces"])


def test_fit_mixture_two_replicas_vs_fp64():
    specs = workloads.fit_mixture(n_replicas=2)
    with Engine(specs) as eng:
        obs = eng.eval()
        states = [eng.state(r) for r in range(len(specs))]
    for r, spec in enumerate(specs):
        _check(spec, obs[r], states[r]["forces"])
