"""Generates tests/golden/spec_*.json + spec_*.npz: the spec dicts the
reference's own Python package builds (``Simulation._native_spec()``) for a few
representative simulations.  Run in a checkout that can import the reference
package (argument: the reference's ``python`` directory); the fixtures, not the
reference, are what the tests use.

    python tests/golden/make_spec_fixtures.py <reference>/python
"""

from __future__ import annotations

import json
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent


def _cases(beads):
    cases = {}

    # Two beads, LJ only (the reference README's minimal example).
    s = beads.System(positions=[[0.25, 0.25, 0.25], [0.75, 0.25, 0.25]], types=[1, 1],
                     box_bound=[[0, 0, 0], [3, 3, 3]], units="nm_kjmol")
    ff = beads.ForceField()
    ff.pair_style("lj", cutoff=0.9)
    ff.pair_coeff("lj", type_i=1, type_j=1, epsilon=1.0, sigma=0.34)
    sim = beads.Simulation(system=s, forcefield=ff, dynamics=beads.Dynamics("velocity_verlet",
                                                                           dt=0.001))
    sim.set_runsteps(10)
    sim.set_thermo(every=5, prefix="minimal")
    sim.set_logging(echo="none")
    cases["minimal"] = sim._native_spec()

    # Binary lattice mixture with Berendsen, neighbour settings, trajectory.
    rng = np.random.default_rng(0)
    g = np.indices((6, 6, 6)).reshape(3, -1).T
    pos = (g + 0.5) * 1.1 + rng.uniform(-0.05, 0.05, g.shape)
    types = (g.sum(axis=1) % 2 + 1).astype(np.int32)
    vel = rng.standard_normal(pos.shape) * 0.5
    s = beads.System(positions=pos, types=types, box_bound=[[0, 0, 0], [6.6, 6.6, 6.6]],
                     velocities=vel, masses=np.where(types == 1, 1.0, 2.0), units="reduced")
    ff = beads.ForceField()
    ff.pair_style("lj", cutoff=2.5, shift=True)
    ff.pair_coeff("lj", type_i=1, type_j=1, epsilon=1.0, sigma=1.0)
    ff.pair_coeff("lj", type_i=1, type_j=2, epsilon=0.7, sigma=0.94)
    ff.pair_coeff("lj", type_i=2, type_j=2, epsilon=0.5, sigma=0.88)
    dyn = beads.Dynamics("velocity_verlet", dt=0.005)
    dyn.set_thermostat("berendsen", temperature=1.0, tau=0.5)
    sim = beads.Simulation(system=s, forcefield=ff, dynamics=dyn)
    sim.set_neighbor(cutoff_buffer=0.3, rebuild_check_every=5, sort_every_rebuild=2,
                     max_neighbors=200)
    sim.set_runsteps(40)
    sim.set_thermo(every=10, prefix="mixture")
    sim.set_trajectory(every=20, prefix="mixture", fields=["tag", "type", "position", "force"])
    sim.save_final_state(prefix="mixture")
    sim.set_logging(echo="log", prefix="mixture")
    cases["mixture"] = sim._native_spec()

    # Bonded chains with angles, dihedrals and explicit exclusions.
    n_chains, beads_per = 4, 12
    pos, bonds, angles, dihs, mol = [], [], [], [], []
    for c in range(n_chains):
        for b in range(beads_per):
            pos.append([1.0 + 0.5 * b, 1.0 + 1.2 * c + (0.1 if b % 2 else -0.1),
                        2.0 + 0.05 * (b % 3)])
            mol.append(c + 1)
        first = c * beads_per + 1
        bonds += [(first + b, first + b + 1, 1) for b in range(beads_per - 1)]
        angles += [(first + b, first + b + 1, first + b + 2, 1) for b in range(beads_per - 2)]
        dihs += [(first + b, first + b + 1, first + b + 2, first + b + 3, 1)
                 for b in range(beads_per - 3)]
    s = beads.System(positions=pos, types=np.ones(len(pos), np.int32),
                     box_bound=[[0, 0, 0], [8.0, 8.0, 6.0]], molecule_ids=mol, units="reduced")
    s.set_topology(bonds=bonds, angles=angles, dihedrals=dihs)
    ff = beads.ForceField()
    ff.pair_style("lj", cutoff=1.12246, shift=True)
    ff.pair_coeff("lj", type_i=1, type_j=1, epsilon=1.0, sigma=1.0)
    ff.bond_style("harmonic")
    ff.bond_coeff("harmonic", type=1, k=500.0, r0=0.5)
    ff.angle_style("harmonic")
    ff.angle_coeff("harmonic", type=1, k=5.0, theta0=150.0)
    ff.dihedral_style("harmonic")
    ff.dihedral_coeff("harmonic", type=1, k=1.0, d=1, n=1)
    ff.exclude_bonded(distance=3)
    sim = beads.Simulation(system=s, forcefield=ff, dynamics=beads.Dynamics("velocity_verlet",
                                                                           dt=0.002))
    sim.set_runsteps(0)
    sim.set_thermo(every=1, prefix="chains")
    sim.set_trajectory(every=1, prefix="chains",
                       fields=["tag", "type", "position", "image", "velocity", "force"])
    sim.set_logging(echo="none")
    cases["chains"] = sim._native_spec()
    return cases


def _split(obj, arrays, path="spec"):
    """JSON-able copy of obj with numpy arrays moved into `arrays`."""
    if isinstance(obj, np.ndarray):
        arrays[path] = obj
        return {"__array__": path}
    if isinstance(obj, dict):
        return {k: _split(v, arrays, f"{path}.{k}") for k, v in obj.items()}
    if isinstance(obj, (list, tuple)):
        return [_split(v, arrays, f"{path}.{i}") for i, v in enumerate(obj)]
    return obj


def main(reference_python: str) -> None:
    sys.path.insert(0, reference_python)
    import beads  # the reference package

    for name, spec in _cases(beads).items():
        arrays: dict = {}
        tree = _split(spec, arrays)
        (HERE / f"spec_{name}.json").write_text(json.dumps(tree, indent=1, sort_keys=True))
        np.savez(HERE / f"spec_{name}.npz", **arrays)
        print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1])
