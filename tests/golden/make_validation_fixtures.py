"""Generates tests/golden/validation_expect.json: for each builder misuse
below, the exception type and message the reference's own Python package
raises (or "ok" when it accepts the call).  The snippets run with ``beads``
bound to the package under test and ``np`` to NumPy; the prelude gives them
valid defaults to spoil one argument at a time.

    python tests/golden/make_validation_fixtures.py <reference>/python
"""

from __future__ import annotations

import json
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent

PRELUDE = '''
BOX = [[0, 0, 0], [6, 6, 6]]
def S(n=2, **kw):
    args = dict(positions=[[0.5 + i, 0.5, 0.5] for i in range(n)], types=[1] * n,
                box_bound=BOX, units="reduced")
    args.update(kw)
    return beads.System(**args)
def CHAIN():
    return S(4)
def FF(types=1):
    ff = beads.ForceField()
    ff.pair_style("lj", cutoff=2.5)
    for a in range(1, types + 1):
        for b in range(a, types + 1):
            ff.pair_coeff("lj", type_i=a, type_j=b, epsilon=1.0, sigma=1.0)
    return ff
def D():
    return beads.Dynamics("velocity_verlet", dt=0.005)
def SIM(system=None, ff=None, dyn=None):
    return beads.Simulation(system=system or S(), forcefield=ff or FF(), dynamics=dyn or D())
'''

CASES = {
    # System
    "system_no_units": "beads.System(positions=[[0.5, 0.5, 0.5]], types=[1], box_bound=BOX)",
    "system_units_type": "S(units=3)",
    "system_units_value": "S(units='si')",
    "system_positions_shape": "S(positions=[[0.5, 0.5], [1.5, 0.5]])",
    "system_positions_empty": "S(positions=np.zeros((0, 3)), types=[])",
    "system_positions_nan": "S(positions=[[0.5, 0.5, 0.5], [np.nan, 0.5, 0.5]])",
    "system_box_shape": "S(box_bound=[[0, 0, 0]])",
    "system_box_inverted": "S(box_bound=[[0, 0, 0], [6, -1, 6]])",
    "system_outside_box": "S(positions=[[0.5, 0.5, 0.5], [6.5, 0.5, 0.5]])",
    "system_types_length": "S(types=[1])",
    "system_types_zero": "S(types=[0, 1])",
    "system_types_gap": "S(types=[1, 3])",
    "system_types_float": "S(types=[1.5, 1])",
    "system_velocities_shape": "S(velocities=[[0, 0, 0]])",
    "system_masses_zero": "S(masses=[0.0, 1.0])",
    "system_masses_shape": "S(masses=[1.0])",
    "system_tags_repeat": "S(tags=[1, 1])",
    "system_tags_range": "S(tags=[1, 3])",
    "system_molecule_gap": "S(molecule_ids=[1, 3])",
    "system_images_shape": "S(images=[[0, 0, 0]])",
    "system_box_missing": "beads.System(positions=[[0.5, 0.5, 0.5]], types=[1], units='reduced')",
    # Topology
    "topology_self_bond": "CHAIN().set_topology(bonds=[(1, 1, 1)])",
    "topology_duplicate_bond": "CHAIN().set_topology(bonds=[(1, 2, 1), (2, 1, 1)])",
    "topology_unknown_tag": "CHAIN().set_topology(bonds=[(1, 9, 1)])",
    "topology_bond_type_zero": "CHAIN().set_topology(bonds=[(1, 2, 0)])",
    "topology_bond_width": "CHAIN().set_topology(bonds=[(1, 2)])",
    "topology_angle_unsupported": "CHAIN().set_topology(bonds=[(1, 2, 1)], angles=[(1, 2, 3, 1)])",
    "topology_dihedral_unsupported": ("CHAIN().set_topology(bonds=[(1, 2, 1), (2, 3, 1)], "
                                      "dihedrals=[(1, 2, 3, 4, 1)])"),
    "topology_type_gap": "CHAIN().set_topology(bonds=[(1, 2, 1), (2, 3, 3)])",
    "topology_after_bind": "s = S(); SIM(system=s); s.set_topology(bonds=[(1, 2, 1)])",
    # ForceField
    "ff_pair_style_unknown": "beads.ForceField().pair_style('morse', cutoff=2.5)",
    "ff_pair_cutoff_negative": "beads.ForceField().pair_style('lj', cutoff=-1.0)",
    "ff_pair_cutoff_missing": "beads.ForceField().pair_style('lj')",
    "ff_pair_cutoff_nan": "beads.ForceField().pair_style('lj', cutoff=float('nan'))",
    "ff_pair_param_unknown": "beads.ForceField().pair_style('lj', cutoff=2.5, colour=1)",
    "ff_pair_coeff_before_style": ("beads.ForceField().pair_coeff('lj', type_i=1, type_j=1, "
                                   "epsilon=1.0, sigma=1.0)"),
    "ff_pair_epsilon_negative": ("ff = beads.ForceField(); ff.pair_style('lj', cutoff=2.5); "
                                 "ff.pair_coeff('lj', type_i=1, type_j=1, epsilon=-1.0, sigma=1.0)"),
    "ff_pair_sigma_zero": ("ff = beads.ForceField(); ff.pair_style('lj', cutoff=2.5); "
                           "ff.pair_coeff('lj', type_i=1, type_j=1, epsilon=1.0, sigma=0.0)"),
    "ff_pair_type_zero": ("ff = beads.ForceField(); ff.pair_style('lj', cutoff=2.5); "
                          "ff.pair_coeff('lj', type_i=0, type_j=1, epsilon=1.0, sigma=1.0)"),
    "ff_pair_coeff_duplicate": ("ff = FF(); "
                                "ff.pair_coeff('lj', type_i=1, type_j=1, epsilon=2.0, sigma=1.0)"),
    "ff_bond_style_unknown": "beads.ForceField().bond_style('fene')",
    "ff_bond_k_negative": ("ff = FF(); ff.bond_style('harmonic'); "
                           "ff.bond_coeff('harmonic', type=1, k=-1.0, r0=1.0)"),
    "ff_bond_coeff_before_style": "FF().bond_coeff('harmonic', type=1, k=1.0, r0=1.0)",
    "ff_angle_theta0_range": ("ff = FF(); ff.angle_style('harmonic'); "
                              "ff.angle_coeff('harmonic', type=1, k=1.0, theta0=200.0)"),
    "ff_dihedral_d": ("ff = FF(); ff.dihedral_style('harmonic'); "
                      "ff.dihedral_coeff('harmonic', type=1, k=1.0, d=2, n=1)"),
    "ff_dihedral_n": ("ff = FF(); ff.dihedral_style('harmonic'); "
                      "ff.dihedral_coeff('harmonic', type=1, k=1.0, d=1, n=-1)"),
    "ff_exclude_distance": "FF().exclude_bonded(distance=4)",
    "ff_pair_style_twice": "ff = FF(); ff.pair_style('lj', cutoff=3.0)",
    # Dynamics
    "dyn_style_unknown": "beads.Dynamics('langevin', dt=0.005)",
    "dyn_dt_zero": "beads.Dynamics('velocity_verlet', dt=0.0)",
    "dyn_dt_negative": "beads.Dynamics('velocity_verlet', dt=-0.005)",
    "dyn_thermostat_unknown": "D().set_thermostat('nose_hoover', temperature=1.0, tau=1.0)",
    "dyn_temperature_negative": "D().set_thermostat('berendsen', temperature=-1.0, tau=1.0)",
    "dyn_tau_zero": "D().set_thermostat('berendsen', temperature=1.0, tau=0.0)",
    # Simulation
    "sim_missing_pair_coeff": "SIM(system=S(types=[1, 2]), ff=FF(1))._native_spec()",
    "sim_runsteps_negative": "SIM().set_runsteps(-1)",
    "sim_runsteps_float": "SIM().set_runsteps(1.5)",
    "sim_thermo_every_zero": "SIM().set_thermo(every=0, prefix='x')",
    "sim_trajectory_field": "SIM().set_trajectory(every=1, prefix='x', fields=['bogus'])",
    "sim_neighbor_skin_negative": "SIM().set_neighbor(cutoff_buffer=-0.1)",
    "sim_neighbor_max_zero": "SIM().set_neighbor(max_neighbors=0)",
    "sim_neighbor_check_zero": "SIM().set_neighbor(rebuild_check_every=0)",
    "sim_logging_echo": "SIM().set_logging(echo='loud')",
    "sim_cutoff_too_large": ("SIM(system=S(box_bound=[[0, 0, 0], [4, 4, 4]]))._native_spec()"),
    "sim_system_type": "beads.Simulation(system=object(), forcefield=FF(), dynamics=D())",
    "sim_valid_spec": "SIM()._native_spec()",
    # Spec building with force fields the builders accepted
    "spec_pair_style_unknown": ("ff = beads.ForceField(); ff.pair_style('morse', cutoff=2.5); "
                                "SIM(ff=ff)._native_spec()"),
    "spec_pair_cutoff_negative": ("ff = beads.ForceField(); ff.pair_style('lj', cutoff=-1.0); "
                                  "ff.pair_coeff('lj', type_i=1, type_j=1, epsilon=1.0, "
                                  "sigma=1.0); SIM(ff=ff)._native_spec()"),
    "spec_pair_cutoff_missing": ("ff = beads.ForceField(); ff.pair_style('lj'); "
                                 "ff.pair_coeff('lj', type_i=1, type_j=1, epsilon=1.0, "
                                 "sigma=1.0); SIM(ff=ff)._native_spec()"),
    "spec_pair_epsilon_negative": ("ff = beads.ForceField(); ff.pair_style('lj', cutoff=2.5); "
                                   "ff.pair_coeff('lj', type_i=1, type_j=1, epsilon=-1.0, "
                                   "sigma=1.0); SIM(ff=ff)._native_spec()"),
    "spec_bond_style_unknown": ("ff = FF(); ff.bond_style('fene'); s = CHAIN(); "
                                "s.set_topology(bonds=[(1, 2, 1)]); "
                                "SIM(system=s, ff=ff)._native_spec()"),
    "spec_bond_k_negative": ("ff = FF(); ff.bond_style('harmonic'); "
                             "ff.bond_coeff('harmonic', type=1, k=-1.0, r0=1.0); s = CHAIN(); "
                             "s.set_topology(bonds=[(1, 2, 1)]); "
                             "SIM(system=s, ff=ff)._native_spec()"),
    "spec_bond_coeff_missing": ("ff = FF(); ff.bond_style('harmonic'); s = CHAIN(); "
                                "s.set_topology(bonds=[(1, 2, 1)]); "
                                "SIM(system=s, ff=ff)._native_spec()"),
    "spec_bond_style_missing": ("s = CHAIN(); s.set_topology(bonds=[(1, 2, 1)]); "
                                "SIM(system=s)._native_spec()"),
    "spec_dihedral_d": ("ff = FF(); ff.bond_style('harmonic'); "
                        "ff.bond_coeff('harmonic', type=1, k=1.0, r0=1.0); "
                        "ff.dihedral_style('harmonic'); "
                        "ff.dihedral_coeff('harmonic', type=1, k=1.0, d=2, n=1); s = CHAIN(); "
                        "s.set_topology(bonds=[(1, 2, 1), (2, 3, 1), (3, 4, 1)], "
                        "dihedrals=[(1, 2, 3, 4, 1)]); SIM(system=s, ff=ff)._native_spec()"),
    "spec_thermostat_negative": ("d = D(); d.set_thermostat('berendsen', temperature=1.0, "
                                 "tau=1.0); SIM(dyn=d)._native_spec()"),
}


def run_case(beads, code: str):
    env = {"beads": beads, "np": np}
    exec(PRELUDE, env)
    try:
        exec(code, env)
    except Exception as exc:  # noqa: BLE001 - recording what the package raises
        return [type(exc).__name__, str(exc)]
    return "ok"


def main(reference_python: str) -> None:
    sys.path.insert(0, reference_python)
    import beads  # the reference's own package

    expect = {name: run_case(beads, code) for name, code in CASES.items()}
    (HERE / "validation_expect.json").write_text(json.dumps(expect, indent=1, sort_keys=True))
    for name, result in sorted(expect.items()):
        print(name, result)


if __name__ == "__main__":
    main(sys.argv[1])
