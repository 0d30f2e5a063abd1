"""The CUDA engine against outputs of the reference engine itself
(tests/golden/ref_*, see tests/test_reference_pin.py)."""

from __future__ import annotations

import numpy as np
import pytest

from beads_b200.engine import Engine, ReplicaSpec
from tests.helpers import rel_rms
from tests.test_reference_pin import CASES, fixture, reference_spread

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", CASES)
def test_engine_forces_vs_reference_fp64(name):
    data, spec = fixture(name)
    r = ReplicaSpec.from_spec(spec)
    with Engine(r) as eng:
        obs = eng.eval()[0]
        forces = eng.state()["forces"]  # tag order
    assert rel_rms(forces, data["forces0_f64"]) <= 1e-5
    header = list(data["thermo_header"])
    row = dict(zip(header, data["thermo0_f64"]))
    for key in ("pair_pe", "bond_pe", "angle_pe", "dihedral_pe", "ke", "temp", "press"):
        if key in row:
            assert abs(obs[key] - row[key]) <= 1e-5 * max(abs(row[key]), 1.0), (key, obs[key],
                                                                              row[key])


@pytest.mark.parametrize("name", CASES)
def test_engine_dynamics_vs_reference(name):
    data, spec = fixture(name)
    r = ReplicaSpec.from_spec(spec)
    steps, every = int(data["md_steps"]), int(data["md_every"])
    rows = []
    with Engine(r) as eng:
        rows.append(eng.eval()[0])
        for _ in range(steps // every):
            rows.append(eng.run(every, every)[0])
        st = eng.state()
    header = list(data["thermo_header"])
    ipe, ike = header.index("pe"), header.index("ke")
    for ours, theirs in zip(rows, data["thermo_f64"]):
        assert ours["step"] == int(theirs[0])
        assert abs(ours["pe"] - theirs[ipe]) <= 1e-4 * max(abs(theirs[ipe]), 1.0)
        assert abs(ours["ke"] - theirs[ike]) <= 1e-4 * max(abs(theirs[ike]), 1.0)
    # Same rebuild policy: same number of neighbour builds as the reference.
    assert rows[-1]["neighbor_build_count"] == int(data["builds_f32"])
    assert rows[-1]["dangerous_rebuild_count"] == int(data["dangerous_f32"])
    length = np.asarray(r.box_bound[1], np.float64) - np.asarray(r.box_bound[0], np.float64)
    unwrapped = st["positions"] + st["images"] * length
    ref_unwrapped = data["final_pos_f64"] + data["final_img_f64"] * length
    # Float coordinates and float pair arithmetic: within a few times the
    # distance between the reference's own float32 and float64 builds.
    assert np.abs(unwrapped - ref_unwrapped).max() < max(1e-4, 4 * reference_spread(data, r))
