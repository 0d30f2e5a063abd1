"""Generates tests/golden/ref_*: outputs of the reference engine itself.

Needs a GPU and the reference's extension modules built by
``python oracle/build_ref.py <reference checkout>`` (float32 and float64
builds).  For each case the spec dict comes from beads_b200's ``Simulation``
(identical to the reference package's, see tests/test_api.py) and is run by
the reference's ``_native.execute_simulation`` twice per precision:

  * runsteps = 0 with a force trajectory and a thermo row: forces, energies,
    virial pressure at the input positions;
  * a short dynamics run: thermo rows, final state, neighbour build counts
    (from the reference's log).

    python tests/golden/make_reference_fixtures.py <output dir> [case ...]
"""

from __future__ import annotations

import pathlib
import re
import sys
import tempfile

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import beads_b200 as beads  # noqa: E402
from beads_b200 import io, workloads  # noqa: E402
from oracle import ref  # noqa: E402


def _system_from(spec_like) -> beads.System:
    s = beads.System(positions=spec_like.positions, types=spec_like.types,
                     box_bound=spec_like.box_bound, velocities=spec_like.velocities,
                     masses=spec_like.masses, tags=spec_like.tags,
                     molecule_ids=spec_like.molecule_ids, images=spec_like.images,
                     units=spec_like.units)
    if spec_like.bonds is not None:
        s.set_topology(bonds=[tuple(map(int, b)) for b in spec_like.bonds],
                       angles=None if spec_like.angles is None
                       else [tuple(map(int, a)) for a in spec_like.angles],
                       dihedrals=None if spec_like.dihedrals is None
                       else [tuple(map(int, d)) for d in spec_like.dihedrals])
    return s


def _forcefield(r) -> beads.ForceField:
    ff = beads.ForceField()
    ff.pair_style("lj", cutoff=float(r.cutoff), shift=bool(r.shift))
    nt = len(r.epsilon)
    for a in range(nt):
        for b in range(a, nt):
            ff.pair_coeff("lj", type_i=a + 1, type_j=b + 1, epsilon=float(r.epsilon[a][b]),
                          sigma=float(r.sigma[a][b]))
    if r.bond_k is not None:
        ff.bond_style("harmonic")
        for t, (k, r0) in enumerate(zip(r.bond_k, r.bond_r0)):
            ff.bond_coeff("harmonic", type=t + 1, k=float(k), r0=float(r0))
    if r.angle_k is not None:
        ff.angle_style("harmonic")
        for t, (k, th) in enumerate(zip(r.angle_k, r.angle_theta0)):
            ff.angle_coeff("harmonic", type=t + 1, k=float(k), theta0=float(th))
    if r.dihedral_k is not None:
        ff.dihedral_style("harmonic")
        for t, (k, d, n) in enumerate(zip(r.dihedral_k, r.dihedral_d, r.dihedral_n)):
            ff.dihedral_coeff("harmonic", type=t + 1, k=float(k), d=int(d), n=int(n))
    if r.exclusion_distance:
        ff.exclude_bonded(distance=int(r.exclusion_distance))
    return ff


def spec_for(r, runsteps: int, prefix: str, *, forces: bool, thermo_every: int) -> dict:
    dyn = beads.Dynamics("velocity_verlet", dt=float(r.dt))
    if r.thermostat is not None:
        dyn.set_thermostat("berendsen", temperature=float(r.thermostat[0]),
                           tau=float(r.thermostat[1]))
    sim = beads.Simulation(system=_system_from(r), forcefield=_forcefield(r), dynamics=dyn)
    sim.set_neighbor(cutoff_buffer=float(r.cutoff_buffer),
                     rebuild_check_every=int(r.rebuild_check_every),
                     sort_every_rebuild=int(r.sort_every_rebuild),
                     max_neighbors=int(r.max_neighbors))
    sim.set_runsteps(runsteps)
    sim.set_thermo(every=thermo_every, prefix=prefix)
    if forces:
        sim.set_trajectory(every=1, prefix=prefix,
                           fields=["tag", "type", "position", "image", "velocity", "force"])
    else:
        sim.save_final_state(prefix=prefix)
    sim.set_logging(echo="log", prefix=prefix)
    return sim._native_spec()


def cases() -> dict:
    lattice = workloads.lj_lattice(n_side=12)
    mixture = workloads.lj_mixture(n=1728, box=(1728 / 20.37) ** (1 / 3), seed=13)
    side = 12
    a = float(mixture.box_bound[1][0]) / side
    g = np.indices((side,) * 3).reshape(3, -1).T.astype(np.float64)
    rng = np.random.default_rng(13)
    mixture.positions = workloads._inside((g + 0.5) * a + rng.uniform(-0.02, 0.02, g.shape),
                                          np.zeros(3), np.full(3, side * a))
    chains = workloads.polymer_melt(n_chains=27, beads=16, seed=17, max_neighbors=128)
    return {"lattice": (lattice, 200, 20), "mixture": (mixture, 200, 20),
            "chains": (chains, 100, 10)}


def _csv(path: pathlib.Path) -> tuple[list[str], np.ndarray]:
    lines = path.read_text().strip().splitlines()
    return lines[0].split(","), np.array([[float(x) for x in ln.split(",")] for ln in lines[1:]])


def _log_value(text: str, key: str) -> str:
    m = re.search(rf"^\s+{key}\s+: (.*)$", text, re.M)
    return m.group(1).strip() if m else ""


def main(out_dir: str, only: list[str]) -> None:
    out = pathlib.Path(out_dir)
    out.mkdir(parents=True, exist_ok=True)
    for name, (r, steps, every) in cases().items():
        if only and name not in only:
            continue
        fixture: dict = {}
        spec0 = spec_for(r, 0, "zero", forces=True, thermo_every=1)
        ref.save_spec(spec0, out / f"ref_{name}_spec.json", out / f"ref_{name}_spec.npz")
        for precision in ("f32", "f64"):
            with tempfile.TemporaryDirectory() as tmp:
                tmp = pathlib.Path(tmp)
                ref.run(precision, spec0, tmp / "zero")
                header, rows = _csv(tmp / "zero" / "zero.thermo.csv")
                traj = io.read_beads_trajectory(tmp / "zero" / "zero.trajectory.beadsbin")
                rec = traj["records"][0]
                order = np.argsort(rec["tag"])
                fixture[f"forces0_{precision}"] = rec["force"][order].astype(np.float64)
                fixture[f"thermo0_{precision}"] = rows[0]
                fixture["thermo_header"] = np.array(header)
                log0 = (tmp / "zero" / "zero.log").read_text()
                fixture["path"] = np.array(_log_value(log0, "path"))
                fixture["excluded_pairs"] = np.array(int(_log_value(log0, "bonded_excluded_pairs")
                                                         or 0))
                spec_md = spec_for(r, steps, "md", forces=False, thermo_every=every)
                ref.run(precision, spec_md, tmp / "md")
                _, rows = _csv(tmp / "md" / "md.thermo.csv")
                fixture[f"thermo_{precision}"] = rows
                state = io.read_state(tmp / "md" / "md.state.beadsbin")
                o = np.argsort(state["tags"])
                fixture[f"final_pos_{precision}"] = state["positions"][o].astype(np.float64)
                fixture[f"final_img_{precision}"] = state["images"][o]
                fixture[f"final_vel_{precision}"] = state["velocities"][o].astype(np.float64)
                log = (tmp / "md" / "md.log").read_text()
                fixture[f"builds_{precision}"] = np.array(int(_log_value(log, "neighbor_build_count")))
                fixture[f"dangerous_{precision}"] = np.array(
                    int(_log_value(log, "dangerous_rebuild_count")))
        fixture["md_steps"] = np.array(steps)
        fixture["md_every"] = np.array(every)
        np.savez_compressed(out / f"ref_{name}.npz", **fixture)
        print("wrote", name, {k: np.shape(v) for k, v in fixture.items()})


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2:])
