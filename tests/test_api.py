"""The reference-compatible Python surface (CPU only).

* The spec dict our ``Simulation`` builds equals, key for key and array for
  array (values and dtypes), the one the reference's own package builds for
  the same inputs (fixtures from tests/golden/make_spec_fixtures.py).
* ``beads_b200._native`` parses the reference's spec dicts.
* Builder validation raises the reference's exception types and messages.
"""

from __future__ import annotations

import json

import numpy as np
import pytest

import beads_b200 as beads
from beads_b200 import _native
from tests.conftest import ROOT

GOLDEN = ROOT / "tests" / "golden"


def load_spec(name: str) -> dict:
    tree = json.loads((GOLDEN / f"spec_{name}.json").read_text())
    arrays = np.load(GOLDEN / f"spec_{name}.npz")

    def join(obj):
        if isinstance(obj, dict):
            if set(obj) == {"__array__"}:
                return arrays[obj["__array__"]]
            return {k: join(v) for k, v in obj.items()}
        if isinstance(obj, list):
            return [join(v) for v in obj]
        return obj

    return join(tree)


def ours_from_spec(spec: dict) -> dict:
    """Rebuilds the same simulation through beads_b200's builders."""
    s = spec["system"]
    system = beads.System(positions=s["positions"], types=s["types"], box_bound=s["box_bound"],
                          velocities=s["velocities"], masses=s["masses"], tags=s["tags"],
                          molecule_ids=s["molecule_ids"], images=s["images"], units=s["units"])
    t = s["topology"]
    if t["bonds"] or t["angles"] or t["dihedrals"]:
        system.set_topology(
            bonds=[(b["tag_i"], b["tag_j"], b["type"]) for b in t["bonds"]],
            angles=[(a["tag_i"], a["tag_j"], a["tag_k"], a["type"]) for a in t["angles"]],
            dihedrals=[(d["tag_i"], d["tag_j"], d["tag_k"], d["tag_l"], d["type"])
                       for d in t["dihedrals"]])
    f = spec["forcefield"]
    ff = beads.ForceField()
    ff.pair_style(f["pair_style"]["style"], **f["pair_style"]["params"])
    for c in f["pair_coeffs"]:
        ff.pair_coeff(c["style"], type_i=c["type_i"], type_j=c["type_j"], **c["params"])
    for kind in ("bond", "angle", "dihedral"):
        if f[f"{kind}_style"] is not None:
            getattr(ff, f"{kind}_style")(f[f"{kind}_style"]["style"],
                                         **f[f"{kind}_style"]["params"])
            for c in f[f"{kind}_coeffs"]:
                getattr(ff, f"{kind}_coeff")(c["style"], type=c["type"], **c["params"])
    if f["bonded_exclusion_policy"] == "explicit":
        ff.exclude_bonded(distance=f["bonded_exclusion_distance"])
    d = spec["dynamics"]
    dyn = beads.Dynamics(d["style"], **d["params"])
    if "thermostat" in d:
        dyn.set_thermostat(d["thermostat"]["style"], **d["thermostat"]["params"])
    sim = beads.Simulation(system=system, forcefield=ff, dynamics=dyn)
    sim.set_neighbor(**spec["neighbor"])
    sim.set_runsteps(spec["runsteps"])
    out = spec["output"]
    if "thermo" in out:
        sim.set_thermo(**out["thermo"])
    if "trajectory" in out:
        sim.set_trajectory(**out["trajectory"])
    if "final_state" in out:
        sim.save_final_state(**out["final_state"])
    sim.set_logging(**out["log"])
    return sim._native_spec()


def assert_same(a, b, path="spec"):
    if isinstance(b, np.ndarray):
        assert isinstance(a, np.ndarray), path
        assert a.dtype == b.dtype and a.shape == b.shape, path
        assert np.array_equal(a, b), path
    elif isinstance(b, dict):
        assert isinstance(a, dict) and set(a) == set(b), (path, sorted(a), sorted(b))
        for k in b:
            assert_same(a[k], b[k], f"{path}.{k}")
    elif isinstance(b, (list, tuple)):
        assert len(a) == len(b), path
        for i, (x, y) in enumerate(zip(a, b)):
            assert_same(x, y, f"{path}[{i}]")
    else:
        assert a == b and type(a) is type(b), (path, a, b)


@pytest.mark.parametrize("name", ["minimal", "mixture", "chains"])
def test_our_spec_equals_reference_spec(name):
    ref = load_spec(name)
    assert_same(ours_from_spec(ref), ref)


@pytest.mark.parametrize("name", ["minimal", "mixture", "chains"])
def test_native_parses_reference_spec(name):
    parsed = _native._Parsed(load_spec(name))
    assert parsed.n == load_spec(name)["system"]["n_particles"]


def test_build_info_is_reference_single_precision():
    assert beads.build_info()["real_dtype"] == "float32"


def _system(**kw):
    base = dict(positions=[[0.5, 0.5, 0.5], [1.5, 0.5, 0.5]], types=[1, 1],
                box_bound=[[0, 0, 0], [4, 4, 4]], units="reduced")
    base.update(kw)
    return beads.System(**base)


@pytest.mark.parametrize("kw, exc, msg", [
    ({"units": None}, TypeError, "explicit units"),
    ({"units": "si"}, ValueError, "units must be"),
    ({"positions": [[5.0, 0.5, 0.5], [1.5, 0.5, 0.5]]}, ValueError, "inside box_bound"),
    ({"types": [1, 3]}, ValueError, "dense one-based"),
    ({"types": [0, 1]}, ValueError, "one-based positive"),
    ({"masses": [1.0, 0.0]}, ValueError, "masses must be"),
    ({"tags": [1, 1]}, ValueError, "permutation"),
    ({"box_bound": [[0, 0, 0], [4, 0, 4]]}, ValueError, "upper row"),
    ({"positions": [[0.5, 0.5, np.nan], [1.5, 0.5, 0.5]]}, ValueError, "finite"),
])
def test_system_validation(kw, exc, msg):
    with pytest.raises(exc, match=msg):
        _system(**kw)


def test_topology_rules():
    s = _system(positions=[[0.5, 0.5, 0.5], [1.5, 0.5, 0.5], [2.5, 0.5, 0.5]], types=[1, 1, 1])
    with pytest.raises(ValueError, match="distinct"):
        s.set_topology(bonds=[(1, 1, 1)])
    with pytest.raises(ValueError, match="duplicate"):
        s.set_topology(bonds=[(1, 2, 1), (2, 1, 1)])
    with pytest.raises(ValueError, match="supporting topology bonds"):
        s.set_topology(bonds=[(1, 2, 1)], angles=[(1, 2, 3, 1)])
    with pytest.raises(ValueError, match="unknown System tag"):
        s.set_topology(bonds=[(1, 9, 1)])
    s.set_topology(bonds=[(2, 1, 1), (3, 2, 1)], angles=[(3, 2, 1, 1)])
    assert s.topology.bonds == ((1, 2, 1), (2, 3, 1))
    assert s.topology.angles == ((1, 2, 3, 1),)


def test_forcefield_and_simulation_rules():
    ff = beads.ForceField()
    with pytest.raises(ValueError, match="pair_style must be set"):
        ff.pair_coeff("lj", type_i=1, type_j=1, epsilon=1.0, sigma=1.0)
    ff.pair_style("lj", cutoff=1.5)
    with pytest.raises(ValueError, match="one active pair_style"):
        ff.pair_style("lj", cutoff=2.0)
    with pytest.raises(ValueError, match="must be 1, 2, or 3"):
        ff.exclude_bonded(distance=4)
    s = _system(types=[1, 2])
    ff.pair_coeff("lj", type_i=1, type_j=1, epsilon=1.0, sigma=1.0)
    with pytest.raises(ValueError, match="missing"):
        beads.Simulation(system=s, forcefield=ff,
                         dynamics=beads.Dynamics("velocity_verlet", dt=0.001))
    with pytest.raises(ValueError, match="exactly parameter"):
        beads.Dynamics("velocity_verlet", dt=0.001, gamma=1.0)
    with pytest.raises(ValueError, match="Unknown Dynamics"):
        beads.Dynamics("langevin", dt=0.001)
    ff2 = beads.ForceField()
    ff2.pair_style("lj", cutoff=1.5)
    ff2.pair_coeff("lj", type_i=1, type_j=1, epsilon=1.0, sigma=1.0)
    sim = beads.Simulation(system=_system(), forcefield=ff2,
                           dynamics=beads.Dynamics("velocity_verlet", dt=0.001))
    with pytest.raises(ValueError, match="requires a prefix"):
        sim.set_logging(echo="log")
    with pytest.raises(ValueError, match="canonical order"):
        sim.set_trajectory(every=1, prefix="x", fields=["tag", "force", "position"])
    with pytest.raises(ValueError, match="cutoff_buffer=0 requires"):
        sim.set_neighbor(cutoff_buffer=0.0, rebuild_check_every=2)


def test_native_rejects_bad_spec_values():
    spec = load_spec("mixture")
    spec["forcefield"]["pair_coeffs"][0]["params"]["epsilon"] = -1.0
    with pytest.raises(ValueError, match="epsilon must be finite and positive"):
        _native._Parsed(spec)
    spec = load_spec("mixture")
    spec["forcefield"]["pair_style"]["style"] = "morse"
    with pytest.raises(ValueError, match="pair_coeff style must match active pair_style"):
        _native._Parsed(spec)
    for coeff in spec["forcefield"]["pair_coeffs"]:
        coeff["style"] = "morse"
    with pytest.raises(ValueError, match='unsupported pair style "morse"'):
        _native._Parsed(spec)
    spec = load_spec("chains")
    spec["forcefield"]["dihedral_coeffs"][0]["params"]["d"] = 2
    with pytest.raises(ValueError, match="must be \\+1 or -1"):
        _native._Parsed(spec)
