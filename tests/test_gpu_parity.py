"""CUDA engine vs the CPU oracle, through the C ABI.

Bars:
  * cell ids and neighbour sets: bit-exact / set-equal;
  * forces: relative RMS vs FP64 <= 1e-5 (FORCE_TOL);
  * energies and virial: relative error <= 1e-5 of the FP64 value, or an
    absolute floor tied to the accumulator resolution;
  * run-to-run and batch-vs-single results: bit-identical.
"""

from __future__ import annotations

import numpy as np
import pytest

from beads_b200 import workloads
from beads_b200.engine import Engine
from tests.helpers import neighbor_sets, oracle_forces, oracle_neighbors, rel_rms

pytestmark = pytest.mark.gpu

FORCE_TOL = 1.0e-5
ENERGY_TOL = 1.0e-5


def _small_mixture(n=12000, seed=11):
    spec = workloads.lj_mixture(n=n, box=(n / 20.37) ** (1 / 3), seed=seed, max_neighbors=160)
    return spec


def _relaxed_mixture(n=12000, seed=11, iters=300):
    spec = _small_mixture(n, seed)
    eng = Engine(spec)
    eng.minimize(iters, 0.004, 200.0)
    st = eng.state()
    eng.close()
    spec.positions = st["positions"]
    return spec


def _small_polymer():
    return workloads.polymer_melt(n_chains=40, beads=50, seed=3, max_neighbors=96)


def test_cell_ids_bit_exact(oracle):
    spec = workloads.lj_lattice()
    with Engine(spec) as eng:
        eng.eval()
        cells = eng.debug_cells()
    expect = oracle.cell_ids(spec.positions, spec.box_bound, spec.cutoff, spec.cutoff_buffer)
    assert np.array_equal(cells, expect)


def test_plan_matches_oracle(oracle):
    for spec in (workloads.lj_lattice(), _small_mixture(), workloads.replica_batch(3, seed=2)[0]):
        with Engine(spec) as eng:
            plan = eng.debug_plan()
        ref = oracle.plan(spec.box_bound, spec.cutoff, spec.cutoff_buffer)
        assert plan["path"] == ref["path"]
        assert np.array_equal(plan["nc"], ref["nc"])


@pytest.mark.parametrize("which", ["lattice", "mixture", "polymer"])
def test_neighbor_sets_equal(oracle, which):
    spec = {"lattice": workloads.lj_lattice, "mixture": _relaxed_mixture,
            "polymer": _small_polymer}[which]()
    with Engine(spec) as eng:
        eng.eval()
        counts, partners = eng.debug_neighbors()
    ocounts, opartners = oracle_neighbors(spec)
    assert np.array_equal(counts, ocounts)
    ours = neighbor_sets(counts, partners)
    theirs = neighbor_sets(ocounts, opartners + 1)
    assert ours == theirs


@pytest.mark.parametrize("which", ["lattice", "mixture", "polymer"])
def test_forces_energy_virial_vs_fp64(which):
    spec = {"lattice": workloads.lj_lattice, "mixture": _relaxed_mixture,
            "polymer": _small_polymer}[which]()
    with Engine(spec) as eng:
        obs = eng.eval()[0]
        st = eng.state()
    f64, e64, w64 = oracle_forces(spec)
    err = rel_rms(st["forces"], f64)
    assert err <= FORCE_TOL, f"force rel RMS {err:.3e}"
    n = spec.n
    floor = 1e-6 * n
    for got, want in ((obs["pair_pe"], e64[0]), (obs["bond_pe"], e64[1]),
                      (obs["angle_pe"], e64[2]), (obs["dihedral_pe"], e64[3]),
                      (obs["virial"], w64)):
        assert abs(got - want) <= max(ENERGY_TOL * abs(want), floor), (got, want)


def test_run_to_run_bit_identical():
    spec = workloads.lj_lattice()
    outs = []
    for _ in range(2):
        with Engine(spec) as eng:
            eng.run(300, 100)
            outs.append(eng.state())
    for key in ("positions", "velocities", "forces", "images"):
        assert np.array_equal(outs[0][key], outs[1][key]), key


def test_batch_matches_single_bitwise():
    specs = workloads.replica_batch(4, n_min=300, n_max=4000, seed=4)
    with Engine(specs) as batch:
        batch.run(50)
        got = [batch.state(r) for r in range(len(specs))]
    for r, spec in enumerate(specs):
        with Engine(spec) as single:
            single.run(50)
            ref = single.state()
        for key in ("positions", "velocities", "forces"):
            assert np.array_equal(got[r][key], ref[key]), (r, key)


def test_short_md_tracks_fp64_oracle(oracle):
    spec = workloads.lj_lattice()
    steps = 50
    with Engine(spec) as eng:
        rows = [eng.eval()[0]]
        for _ in range(steps // 10):
            rows.append(eng.run(10, 10)[0])
        st = eng.state()
    from tests.helpers import oracle_ff

    pos, vel, img, thermo, builds = oracle.md(
        spec.positions, spec.velocities, spec.masses, spec.types, spec.box_bound,
        oracle_ff(spec), dt=spec.dt, steps=steps, skin=spec.cutoff_buffer,
        check_every=spec.rebuild_check_every, obs_every=10)
    for ours, ref in zip(rows, thermo):
        assert ours["step"] == int(ref[0])
        etot = ours["pe"] + ours["ke"]
        eref = ref[1] + ref[5]
        assert abs(etot - eref) <= 2e-5 * abs(eref) + 1e-3, (ours["step"], etot, eref)
    unwrapped = st["positions"] + st["images"] * (spec.box_bound[1] - spec.box_bound[0])
    ref_unwrapped = pos + img * (spec.box_bound[1] - spec.box_bound[0])
    assert np.abs(unwrapped - ref_unwrapped).max() < 1e-3


def test_energy_conservation_nve():
    # Shifted LJ keeps U continuous at rc, so the total energy only moves by
    # integration error (plus the small force step at rc).
    spec = workloads.lj_lattice()
    spec.shift = True
    with Engine(spec) as eng:
        eng.run(500)  # melt the lattice first
        rows = [eng.run(100, 100)[0] for _ in range(10)]
    etot = np.array([r["pe"] + r["ke"] for r in rows])
    drift = np.ptp(etot) / spec.n
    assert drift < 2e-3, drift


def test_berendsen_moves_temperature_toward_target():
    spec = workloads.lj_lattice(temperature=2.0)
    spec.thermostat = (1.0, 0.1)
    with Engine(spec) as eng:
        t0 = eng.eval()[0]["temp"]
        rows = [eng.run(100, 100)[0] for _ in range(6)]
    assert abs(rows[-1]["temp"] - 1.0) < abs(t0 - 1.0)
    assert abs(rows[-1]["temp"] - 1.0) < 0.15


def test_neighbor_overflow_raises():
    spec = workloads.lj_lattice()
    spec.max_neighbors = 20
    with Engine(spec) as eng:
        with pytest.raises(RuntimeError, match="NeighborList overflow"):
            eng.eval()


@pytest.mark.parametrize("box", [6.2, 9.0])
def test_direct_and_small_dimension_paths(oracle, box):
    rng = np.random.default_rng(5)
    # box 6.2 with rc+skin 2.8 -> 2 cells per axis (direct path);
    # 9.0 x 6.2 x 9.0 -> mixed counts (small-dimension path).
    lens = np.array([box, 6.2, box])
    n = int(0.8 * lens.prod())
    g = np.indices((12, 12, 12)).reshape(3, -1).T[:n] / 12.0
    pos = (g * lens + rng.uniform(-0.01, 0.01, g.shape)) % lens
    spec = workloads.lj_lattice()
    spec.positions = pos.astype(np.float32)
    spec.types = np.ones(n, np.int32)
    spec.velocities = np.zeros((n, 3), np.float32)
    spec.masses = np.ones(n, np.float32)
    spec.box_bound = np.array([[0, 0, 0], lens], np.float32)
    with Engine(spec) as eng:
        eng.eval()
        plan = eng.debug_plan()
        counts, partners = eng.debug_neighbors()
        st = eng.state()
    assert plan["path"] == ("direct" if box < 8 else "small_dimension")
    ocounts, opartners = oracle_neighbors(spec)
    assert neighbor_sets(counts, partners) == neighbor_sets(ocounts, opartners + 1)
    f64, _, _ = oracle_forces(spec)
    assert rel_rms(st["forces"], f64) <= FORCE_TOL


def test_exclusions_remove_bonded_pairs():
    spec = _small_polymer()
    with Engine(spec) as eng:
        eng.eval()
        counts, partners = eng.debug_neighbors()
    sets = neighbor_sets(counts, partners)
    # 1-2 and 1-3 partners along a chain never appear (exclusion distance 2).
    beads = 50
    for t in range(1, spec.n + 1):
        row = set(sets[t - 1])
        chain0 = (t - 1) // beads
        for d in (1, 2):
            for u in (t - d, t + d):
                if 1 <= u <= spec.n and (u - 1) // beads == chain0:
                    assert u not in row


@pytest.mark.parametrize("density", [3.0, 10.0])
def test_crowded_cells_sort_and_list(oracle, density):
    """Cells far above a warp's 32 slots: ~90 per cell goes through the
    shared-memory rank sort, ~300 through the insertion sort.  The lists
    must equal the oracle's sets, and a second build of the same state must
    give the same entries in the same order."""
    rng = np.random.default_rng(int(density))
    lens = np.array([6.2, 6.2, 6.2])
    n = int(density * lens.prod())
    side = int(np.ceil(n ** (1 / 3)))
    a = 6.2 / side
    g = np.indices((side,) * 3).reshape(3, -1).T[rng.permutation(side ** 3)[:n]]
    # A jittered lattice: crowded cells without overlapping pairs.
    pos = (g + 0.5 + rng.uniform(-0.1, 0.1, g.shape)) * a
    spec = workloads.lj_lattice()
    spec.positions = pos.astype(np.float32)
    spec.types = np.ones(n, np.int32)
    spec.velocities = np.zeros((n, 3), np.float32)
    spec.masses = np.ones(n, np.float32)
    spec.box_bound = np.array([[0, 0, 0], lens], np.float32)
    spec.max_neighbors = 1024
    with Engine(spec) as eng:
        eng.eval()
        counts, partners = eng.debug_neighbors()
        eng.eval()
        counts2, partners2 = eng.debug_neighbors()
    ocounts, opartners = oracle_neighbors(spec)
    assert np.array_equal(counts, ocounts)
    assert neighbor_sets(counts, partners) == neighbor_sets(ocounts, opartners + 1)
    assert np.array_equal(counts, counts2) and np.array_equal(partners, partners2)


@pytest.mark.parametrize("distance", [1, 3])
def test_exclusion_distances_match_oracle(oracle, distance):
    """Bond-graph exclusions at distance 1 (one partner row entry per bond)
    and 3 (up to six partners along a chain): the list build's exclusion
    check against the oracle's neighbour sets."""
    spec = workloads.polymer_melt(n_chains=40, beads=50, seed=3, max_neighbors=96,
                                  exclusion_distance=distance)
    with Engine(spec) as eng:
        eng.eval()
        counts, partners = eng.debug_neighbors()
    ocounts, opartners = oracle_neighbors(spec)
    assert np.array_equal(counts, ocounts)
    assert neighbor_sets(counts, partners) == neighbor_sets(ocounts, opartners + 1)
