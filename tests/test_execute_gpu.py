"""execute_simulation end to end on the GPU: the reference's spec dicts in,
the reference's files out (thermo CSV, BEADS_TRAJECTORY, BEADS_SNAPSHOT, log),
with values checked against the CPU oracle."""

from __future__ import annotations

import numpy as np
import pytest

import beads_b200 as beads
from beads_b200 import _native, io
from oracle import oracle as O
from tests.test_api import load_spec

pytestmark = pytest.mark.gpu


def _oracle_ff(spec):
    f = spec["forcefield"]
    nt = int(spec["system"]["types"].max())
    eps = np.zeros((nt, nt))
    sig = np.zeros((nt, nt))
    for c in f["pair_coeffs"]:
        a, b = c["type_i"] - 1, c["type_j"] - 1
        eps[a, b] = eps[b, a] = c["params"]["epsilon"]
        sig[a, b] = sig[b, a] = c["params"]["sigma"]
    kw = {}
    if f["bond_style"]:
        kw["bond_k"] = [c["params"]["k"] for c in f["bond_coeffs"]]
        kw["bond_r0"] = [c["params"]["r0"] for c in f["bond_coeffs"]]
    if f["angle_style"]:
        kw["angle_k"] = [c["params"]["k"] for c in f["angle_coeffs"]]
        kw["angle_theta0"] = [c["params"]["theta0"] for c in f["angle_coeffs"]]
    if f["dihedral_style"]:
        kw["dihedral_k"] = [c["params"]["k"] for c in f["dihedral_coeffs"]]
        kw["dihedral_d"] = [c["params"]["d"] for c in f["dihedral_coeffs"]]
        kw["dihedral_n"] = [c["params"]["n"] for c in f["dihedral_coeffs"]]
    return O.ForceField(epsilon=eps.ravel(), sigma=sig.ravel(),
                        cutoff=f["pair_style"]["params"]["cutoff"],
                        shift=f["pair_style"]["params"].get("shift", False),
                        exclusion_distance=f["bonded_exclusion_distance"] or 0, **kw)


def _oracle_step0(spec):
    s = spec["system"]
    order = np.argsort(s["tags"])  # oracle rows are tag order
    t = s["topology"]
    return O.forces(s["positions"][order], s["types"][order], s["box_bound"], _oracle_ff(spec),
                    skin=spec["neighbor"]["cutoff_buffer"],
                    bonds=[(b["tag_i"], b["tag_j"], b["type"]) for b in t["bonds"]],
                    angles=[(a["tag_i"], a["tag_j"], a["tag_k"], a["type"]) for a in t["angles"]],
                    dihedrals=[(d["tag_i"], d["tag_j"], d["tag_k"], d["tag_l"], d["type"])
                               for d in t["dihedrals"]])


def _read_csv(path):
    lines = path.read_text().strip().splitlines()
    header = lines[0].split(",")
    rows = [dict(zip(header, map(float, line.split(",")))) for line in lines[1:]]
    return header, rows, lines


def _run(spec, tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    _native.execute_simulation(spec)


def test_chains_zero_step_files_match_oracle(tmp_path, monkeypatch):
    spec = load_spec("chains")
    _run(spec, tmp_path, monkeypatch)
    header, rows, lines = _read_csv(tmp_path / "chains.thermo.csv")
    assert header == ["step", "pe", "pair_pe", "bond_pe", "angle_pe", "dihedral_pe", "ke",
                      "temp", "press"]
    assert [r["step"] for r in rows] == [0.0]
    f64, e64, w64 = _oracle_step0(spec)
    row = rows[0]
    for key, want in zip(("pair_pe", "bond_pe", "angle_pe", "dihedral_pe"), e64):
        assert abs(row[key] - want) <= 1e-5 * max(abs(want), 1.0), (key, row[key], want)
    traj = io.read_beads_trajectory(tmp_path / "chains.trajectory.beadsbin")
    assert traj["fields"] == ["tag", "type", "position", "image", "velocity", "force"]
    assert traj["frame_count"] == 1 and int(traj["steps"][0]) == 0
    rec = traj["records"][0]
    order = np.argsort(rec["tag"])
    forces = rec["force"][order].astype(np.float64)
    err = np.sqrt(((forces - f64) ** 2).sum() / (f64 ** 2).sum())
    assert err <= 1e-5, err
    s = spec["system"]
    assert np.array_equal(rec["position"][order], s["positions"][np.argsort(s["tags"])])


def test_mixture_run_writes_reference_formats(tmp_path, monkeypatch):
    spec = load_spec("mixture")
    _run(spec, tmp_path, monkeypatch)
    header, rows, lines = _read_csv(tmp_path / "mixture.thermo.csv")
    assert header == ["step", "pe", "pair_pe", "ke", "temp", "press"]
    assert [int(r["step"]) for r in rows] == [0, 10, 20, 30, 40]
    # 9 significant digits, as the reference's setprecision(9) stream writes.
    for tok in lines[1].split(",")[1:]:
        mantissa = tok.split("e")[0].lstrip("-")
        assert len(mantissa.replace(".", "").lstrip("0")) <= 9, tok
    f64, e64, w64 = _oracle_step0(spec)
    r0 = rows[0]
    assert abs(r0["pair_pe"] - e64[0]) <= 1e-5 * abs(e64[0])
    s = spec["system"]
    v = s["velocities"].astype(np.float64)
    ke = 0.5 * (s["masses"][:, None] * v * v).sum()
    assert abs(r0["ke"] - ke) <= 1e-6 * ke
    dof = 3 * s["n_particles"] - 3
    assert abs(r0["temp"] - 2 * ke / dof) <= 1e-6 * r0["temp"]
    vol = np.prod(s["box_bound"][1] - s["box_bound"][0])
    assert abs(r0["press"] - (2 * ke + w64) / (3 * vol)) <= 1e-5 * max(abs(r0["press"]), 1.0)
    traj = io.read_beads_trajectory(tmp_path / "mixture.trajectory.beadsbin")
    assert traj["fields"] == ["tag", "type", "position", "force"]
    assert [int(x) for x in traj["steps"]] == [0, 20, 40]
    assert traj["units"] == "reduced" and traj["record_bytes"] == 4 + 4 + 12 + 12
    state = io.read_state(tmp_path / "mixture.state.beadsbin")
    assert state["units"] == "reduced"
    restored = beads.System.from_state(tmp_path / "mixture.state.beadsbin")
    assert restored.n_particles == s["n_particles"]
    last = traj["records"][-1]
    o1 = np.argsort(last["tag"])
    o2 = np.argsort(state["tags"])
    assert np.array_equal(last["position"][o1], state["positions"][o2])
    log = (tmp_path / "mixture.log").read_text()
    for needle in ("execute start", "neighbor summary", "execute end", "neighbor_build_count",
                   "steps_per_second", "THERMO"):
        assert needle in log


def test_minimal_readme_example(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    s = beads.System(positions=[[0.25, 0.25, 0.25], [0.75, 0.25, 0.25]], types=[1, 1],
                     box_bound=[[0, 0, 0], [3, 3, 3]], units="nm_kjmol")
    ff = beads.ForceField()
    ff.pair_style("lj", cutoff=0.9)
    ff.pair_coeff("lj", type_i=1, type_j=1, epsilon=1.0, sigma=0.34)
    sim = beads.Simulation(system=s, forcefield=ff,
                           dynamics=beads.Dynamics("velocity_verlet", dt=0.001))
    sim.set_runsteps(10)
    sim.set_thermo(every=5, prefix="minimal")
    sim.set_logging(echo="none")
    sim.execute()
    header, rows, _ = _read_csv(tmp_path / "minimal.thermo.csv")
    assert [int(r["step"]) for r in rows] == [0, 5, 10]
    with pytest.raises(RuntimeError, match="cannot be called after execute"):
        sim.execute()


def test_neighbor_overflow_is_runtime_error(tmp_path, monkeypatch):
    spec = load_spec("mixture")
    spec["neighbor"]["max_neighbors"] = 10
    with pytest.raises(RuntimeError, match="NeighborList overflow"):
        _run(spec, tmp_path, monkeypatch)
