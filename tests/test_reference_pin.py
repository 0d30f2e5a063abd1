"""The CPU oracle pinned against outputs of the reference engine itself.

tests/golden/ref_<case>.npz hold what the reference's own extension module
(float32 and float64 builds, oracle/build_ref.py) wrote for the input in
ref_<case>_spec.{json,npz} (tests/golden/make_reference_fixtures.py):
step-0 forces and thermo row, a short dynamics run's thermo rows, final
state and neighbour build counts, the neighbour path and the bonded
exclusion count from its log.
"""

from __future__ import annotations

import copy

import numpy as np
import pytest

from beads_b200.engine import ReplicaSpec
from oracle import oracle as O
from oracle import ref
from tests.conftest import ROOT
from tests.helpers import oracle_ff, rel_rms

GOLDEN = ROOT / "tests" / "golden"
CASES = ["lattice", "mixture", "chains"]


def fixture(name: str):
    data = np.load(GOLDEN / f"ref_{name}.npz")
    spec = ref.load_spec(GOLDEN / f"ref_{name}_spec.json", GOLDEN / f"ref_{name}_spec.npz")
    return data, spec


def tag_ordered(spec: dict) -> ReplicaSpec:
    r = ReplicaSpec.from_spec(spec)
    order = np.argsort(r.tags)
    r = copy.copy(r)
    for key in ("positions", "types", "velocities", "masses", "molecule_ids", "images"):
        setattr(r, key, np.asarray(getattr(r, key))[order])
    r.tags = None
    return r


def reference_spread(data, r) -> float:
    """Largest final-position difference between the reference's float32 and
    float64 builds after the fixture's dynamics run (unwrapped)."""
    length = np.asarray(r.box_bound[1], np.float64) - np.asarray(r.box_bound[0], np.float64)
    a = data["final_pos_f32"] + data["final_img_f32"] * length
    b = data["final_pos_f64"] + data["final_img_f64"] * length
    return float(np.abs(a - b).max())


def _kinetic(vel, masses):
    v = np.asarray(vel, np.float64)
    return 0.5 * float((np.asarray(masses, np.float64)[:, None] * v * v).sum())


@pytest.mark.parametrize("name", CASES)
def test_oracle_forces_match_reference_fp64(name):
    data, spec = fixture(name)
    r = tag_ordered(spec)
    f64, energies, virial = O.forces(r.positions, r.types, r.box_bound, oracle_ff(r),
                                     skin=r.cutoff_buffer, bonds=r.bonds, angles=r.angles,
                                     dihedrals=r.dihedrals)
    # Both are double precision; they differ by summation order only.
    assert rel_rms(f64, data["forces0_f64"]) < 1e-9
    header = list(data["thermo_header"])
    row = dict(zip(header, data["thermo0_f64"]))
    parts = {"pair_pe": energies[0], "bond_pe": energies[1], "angle_pe": energies[2],
             "dihedral_pe": energies[3]}
    for key, want in parts.items():
        if key in row:  # the CSV holds 9 significant digits
            assert abs(row[key] - want) <= 2e-8 * max(abs(want), 1.0), (key, row[key], want)
    vol = float(np.prod(np.asarray(r.box_bound[1], np.float64) - r.box_bound[0]))
    ke = _kinetic(r.velocities, r.masses)
    scale = 16.60539067 if r.units == "nm_kjmol" else 1.0
    press = scale * (2 * ke + virial) / (3 * vol)
    assert abs(row["press"] - press) <= 2e-8 * max(abs(press), 1.0)


@pytest.mark.parametrize("name", CASES)
def test_reference_float32_build_force_error(name):
    """The reference's own single-precision build against its double build:
    the error level its users see (recorded, and bounded)."""
    data, _ = fixture(name)
    assert rel_rms(data["forces0_f32"], data["forces0_f64"]) < 1e-4


@pytest.mark.parametrize("name", CASES)
def test_plan_and_exclusions_match_reference(name):
    data, spec = fixture(name)
    r = tag_ordered(spec)
    assert O.plan(r.box_bound, r.cutoff, r.cutoff_buffer)["path"] == str(data["path"])
    n_excl = (len(O.exclusion_pairs(r.n, r.bonds, r.exclusion_distance))
              if r.exclusion_distance and r.bonds is not None else 0)
    assert n_excl == int(data["excluded_pairs"])


@pytest.mark.parametrize("name", CASES)
def test_oracle_dynamics_track_reference_fp64(name):
    data, spec = fixture(name)
    r = tag_ordered(spec)
    steps, every = int(data["md_steps"]), int(data["md_every"])
    kt = None
    if r.thermostat is not None:
        kb = 0.00831446261815324 if r.units == "nm_kjmol" else 1.0
        kt = kb * float(np.float32(r.thermostat[0]))
    pos, vel, img, rows, builds = O.md(
        r.positions, r.velocities, r.masses, r.types, r.box_bound, oracle_ff(r), dt=r.dt,
        steps=steps, skin=r.cutoff_buffer, check_every=r.rebuild_check_every, bonds=r.bonds,
        angles=r.angles, dihedrals=r.dihedrals, thermostat=r.thermostat is not None,
        kt_target=kt or 0.0, tau=float(np.float32(r.thermostat[1])) if kt else 1.0,
        obs_every=every)
    ref_rows = data["thermo_f64"]
    header = list(data["thermo_header"])
    ipe, ike = header.index("pe"), header.index("ke")
    for ours, theirs in zip(rows, ref_rows):
        assert int(ours[0]) == int(theirs[0])
        pe = ours[1] + ours[2] + ours[3] + ours[4]
        assert abs(pe - theirs[ipe]) <= 1e-5 * max(abs(theirs[ipe]), 1.0)
        assert abs(ours[5] - theirs[ike]) <= 1e-5 * max(abs(theirs[ike]), 1.0)
    assert builds == int(data["builds_f64"])
    length = np.asarray(r.box_bound[1], np.float64) - r.box_bound[0]
    unwrapped = pos + img * length
    ref_unwrapped = data["final_pos_f64"] + data["final_img_f64"] * length
    # The oracle evaluates forces at float-rounded coordinates, so after a few
    # hundred chaotic steps it sits as far from the reference's double build
    # as the reference's own float build does.
    assert np.abs(unwrapped - ref_unwrapped).max() < max(1e-4, 2 * reference_spread(data, r))
