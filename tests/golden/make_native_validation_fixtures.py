"""Generates tests/golden/native_validation_expect.json: for each simulation
below that the Python builders accept but the native layer must refuse, the
exception type and message of the reference's own compiled
``_native.execute_simulation`` (the float32 module oracle/build_ref.py
builds; it validates the spec before touching the GPU).  The snippets build a
spec dict with ``beads`` bound to the package under test; ``edit(spec)``
cases then change one entry of the dict directly.

    python tests/golden/make_native_validation_fixtures.py <reference checkout>
"""

from __future__ import annotations

import importlib.util
import json
import os
import pathlib
import sys
import tempfile

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
from make_validation_fixtures import PRELUDE  # noqa: E402

SPEC = "spec = SIM(ff=ff)._native_spec()"
LJ = "ff = beads.ForceField(); ff.pair_style('lj', cutoff={cut}); "
COEFF = "ff.pair_coeff('lj', type_i=1, type_j=1, epsilon={eps}, sigma={sig}); "

CASES = {
    "pair_epsilon_negative": LJ.format(cut=2.5) + COEFF.format(eps=-1.0, sig=1.0) + SPEC,
    "pair_sigma_zero": LJ.format(cut=2.5) + COEFF.format(eps=1.0, sig=0.0) + SPEC,
    "pair_cutoff_negative": LJ.format(cut=-1.0) + COEFF.format(eps=1.0, sig=1.0) + SPEC,
    "cutoff_beyond_half_box": (LJ.format(cut=2.9) + COEFF.format(eps=1.0, sig=1.0) +
                               "spec = SIM(ff=ff)._native_spec()"),
    "bond_k_negative": ("ff = FF(); ff.bond_style('harmonic'); "
                        "ff.bond_coeff('harmonic', type=1, k=-1.0, r0=1.0); s = CHAIN(); "
                        "s.set_topology(bonds=[(1, 2, 1)]); "
                        "spec = SIM(system=s, ff=ff)._native_spec()"),
    "bond_r0_negative": ("ff = FF(); ff.bond_style('harmonic'); "
                         "ff.bond_coeff('harmonic', type=1, k=1.0, r0=-1.0); s = CHAIN(); "
                         "s.set_topology(bonds=[(1, 2, 1)]); "
                         "spec = SIM(system=s, ff=ff)._native_spec()"),
    "angle_theta0_range": ("ff = FF(); ff.bond_style('harmonic'); "
                           "ff.bond_coeff('harmonic', type=1, k=1.0, r0=1.0); "
                           "ff.angle_style('harmonic'); "
                           "ff.angle_coeff('harmonic', type=1, k=1.0, theta0=200.0); s = CHAIN(); "
                           "s.set_topology(bonds=[(1, 2, 1), (2, 3, 1)], angles=[(1, 2, 3, 1)]); "
                           "spec = SIM(system=s, ff=ff)._native_spec()"),
    "dihedral_d": ("ff = FF(); ff.bond_style('harmonic'); "
                   "ff.bond_coeff('harmonic', type=1, k=1.0, r0=1.0); "
                   "ff.dihedral_style('harmonic'); "
                   "ff.dihedral_coeff('harmonic', type=1, k=1.0, d=2, n=1); s = CHAIN(); "
                   "s.set_topology(bonds=[(1, 2, 1), (2, 3, 1), (3, 4, 1)], "
                   "dihedrals=[(1, 2, 3, 4, 1)]); spec = SIM(system=s, ff=ff)._native_spec()"),
    "dihedral_n": ("ff = FF(); ff.bond_style('harmonic'); "
                   "ff.bond_coeff('harmonic', type=1, k=1.0, r0=1.0); "
                   "ff.dihedral_style('harmonic'); "
                   "ff.dihedral_coeff('harmonic', type=1, k=1.0, d=1, n=-1); s = CHAIN(); "
                   "s.set_topology(bonds=[(1, 2, 1), (2, 3, 1), (3, 4, 1)], "
                   "dihedrals=[(1, 2, 3, 4, 1)]); spec = SIM(system=s, ff=ff)._native_spec()"),
    "positions_float64": ("spec = SIM()._native_spec(); "
                          "spec['system']['positions'] = "
                          "spec['system']['positions'].astype(np.float64)"),
    "positions_not_contiguous": ("spec = SIM()._native_spec(); p = spec['system']['positions']; "
                                 "spec['system']['positions'] = np.asfortranarray(np.concatenate("
                                 "[p, p])[::2])"),
    "types_wrong_dtype": ("spec = SIM()._native_spec(); "
                          "spec['system']['types'] = spec['system']['types'].astype(np.int64)"),
    "runsteps_negative": "spec = SIM()._native_spec(); spec['runsteps'] = -1",
    "runsteps_float": "spec = SIM()._native_spec(); spec['runsteps'] = 1.5",
    "n_particles_mismatch": "spec = SIM()._native_spec(); spec['system']['n_particles'] = 3",
    "masses_shape": ("spec = SIM()._native_spec(); "
                     "spec['system']['masses'] = np.ones(3, np.float32)"),
    "tags_dtype": ("spec = SIM()._native_spec(); "
                   "spec['system']['tags'] = spec['system']['tags'].astype(np.int32)"),
    "images_shape": ("spec = SIM()._native_spec(); "
                     "spec['system']['images'] = np.zeros((2, 2), np.int32)"),
    "box_bound_shape": ("spec = SIM()._native_spec(); "
                        "spec['system']['box_bound'] = np.zeros((3, 2), np.float32)"),
    "neighbor_missing": "spec = SIM()._native_spec(); del spec['neighbor']",
    "max_neighbors_zero": "spec = SIM()._native_spec(); spec['neighbor']['max_neighbors'] = 0",
    "cutoff_buffer_negative": ("spec = SIM()._native_spec(); "
                               "spec['neighbor']['cutoff_buffer'] = -0.1"),
    "dynamics_style": "spec = SIM()._native_spec(); spec['dynamics']['style'] = 'langevin'",
    "pair_style_unknown": ("spec = SIM()._native_spec(); "
                           "spec['forcefield']['pair_style']['style'] = 'morse'"),
    "log_echo": "spec = SIM()._native_spec(); spec['output']['log']['echo'] = 'loud'",
    "system_missing": "spec = SIM()._native_spec(); del spec['system']",
    "dt_zero": "spec = SIM()._native_spec(); spec['dynamics']['params']['dt'] = 0.0",
    "units_unknown": "spec = SIM()._native_spec(); spec['system']['units'] = 'si'",
}


def native_error(execute, spec: dict):
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.chdir(tmp)
        try:
            execute(spec)
        except Exception as exc:  # noqa: BLE001 - recording what the engine raises
            return [type(exc).__name__, str(exc)]
        finally:
            os.chdir(cwd)
    return "ok"


def build_spec(beads, code: str) -> dict:
    env = {"beads": beads, "np": np}
    exec(PRELUDE, env)
    exec(code, env)
    return env["spec"]


def main(reference: str) -> None:
    ref_root = pathlib.Path(reference)
    sys.path.insert(0, str(ref_root / "python"))
    import beads  # the reference's own package

    repo = HERE.parents[1]
    sys.path.insert(0, str(repo))
    from oracle import ref

    loader = importlib.util.spec_from_file_location("_native", ref.module_path("f32"))
    native = importlib.util.module_from_spec(loader)
    loader.loader.exec_module(native)
    expect = {}
    for name, code in CASES.items():
        result = native_error(native.execute_simulation, build_spec(beads, code))
        # Keep only refusals of the spec itself, not the missing GPU here.
        if result == "ok" or "CUDA" in result[1] or "cuda" in result[1]:
            print("skipped", name, result)
            continue
        expect[name] = result
        print(name, result)
    (HERE / "native_validation_expect.json").write_text(json.dumps(expect, indent=1,
                                                                   sort_keys=True))


if __name__ == "__main__":
    main(sys.argv[1])
