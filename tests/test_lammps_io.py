"""LAMMPS data import and dump export against what the reference's own
``beads.io`` made of the same files (tests/golden/lammps, written by
tests/golden/make_lammps_fixtures.py)."""

from __future__ import annotations

import json

import numpy as np
import pytest

from beads_b200 import io
from tests.conftest import ROOT

GOLDEN = ROOT / "tests" / "golden" / "lammps"
EXPECT = json.loads((GOLDEN / "expect.json").read_text())


@pytest.mark.parametrize("name", sorted(EXPECT["valid"]))
def test_read_lammps_data_matches_reference(name):
    system = io.read_lammps_data(GOLDEN / f"{name}.data", units="reduced")
    ref = np.load(GOLDEN / f"{name}.npz")
    for key in ("positions", "box_bound", "types", "velocities", "masses", "tags",
                "molecule_ids", "images"):
        ours = np.asarray(getattr(system, key))
        assert ours.dtype == ref[key].dtype, key
        assert np.array_equal(ours, ref[key]), key
    topo = EXPECT["valid"][name]
    assert [list(b) for b in system.topology.bonds] == topo["bonds"]
    assert [list(a) for a in system.topology.angles] == topo["angles"]
    assert [list(d) for d in system.topology.dihedrals] == topo["dihedrals"]


@pytest.mark.parametrize("name", sorted(EXPECT["invalid"]))
def test_read_lammps_data_rejects_like_reference(name):
    kind, message = EXPECT["invalid"][name]
    with pytest.raises({"ValueError": ValueError, "TypeError": TypeError}[kind]) as err:
        io.read_lammps_data(GOLDEN / f"bad_{name}.data", units="reduced")
    assert str(err.value) == message


def test_read_lammps_data_requires_units():
    with pytest.raises(TypeError):
        io.read_lammps_data(GOLDEN / "plain.data", units=None)


@pytest.mark.parametrize("label", sorted(EXPECT["dumps"]))
def test_write_lammps_dump_matches_reference(tmp_path, label):
    out = tmp_path / "out.dump"
    io.write_lammps_dump(GOLDEN / "traj.beadsbin", out, **EXPECT["dumps"][label])
    assert out.read_text() == (GOLDEN / f"{label}.dump").read_text()


@pytest.mark.parametrize("kwargs, exc", [({"precision": 0}, ValueError),
                                         ({"precision": 18}, ValueError),
                                         ({"precision": True}, TypeError),
                                         ({"precision": 2.5}, TypeError),
                                         ({"sort_by_tag": 1}, TypeError)])
def test_write_lammps_dump_argument_checks(tmp_path, kwargs, exc):
    with pytest.raises(exc):
        io.write_lammps_dump(GOLDEN / "traj.beadsbin", tmp_path / "x.dump", **kwargs)
