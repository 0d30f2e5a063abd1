"""The C-ABI library loads and exports every entry point include/beads_b200.h
declares, and refuses invalid replicas before any device work (no compute
call: this runs without a GPU)."""

from __future__ import annotations

import ctypes
import re

import pytest

from tests.conftest import ROOT


def declared_symbols() -> set[str]:
    text = (ROOT / "include" / "beads_b200.h").read_text()
    return set(re.findall(r"BEADS_API\s+(?:int|void)\s+(beads_\w+)\s*\(", text))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert {"beads_execute", "beads_build_info", "beads_batch_create", "beads_run"} <= names


def test_library_exports_every_declared_symbol(native):
    lib = ctypes.CDLL(str(ROOT / "beads_b200" / "libbeads_b200.so"))
    missing = [name for name in sorted(declared_symbols()) if not hasattr(lib, name)]
    assert not missing, missing


def test_build_info_matches_reference_keys():
    from beads_b200 import _lib

    info = _lib.build_info()
    assert info == {
        "real_precision": "single",
        "real_dtype": "float32",
        "type_dtype": "int32",
        "index_dtype": "uint32",
        "image_dtype": "int32",
        "runstep_dtype": "uint64",
    }


def test_python_binding_lists_every_symbol():
    from beads_b200 import _lib

    assert set(_lib.EXPORTED) == declared_symbols()


def test_invalid_input_is_rejected_before_any_device_work():
    import numpy as np

    from beads_b200.engine import Engine, ReplicaSpec

    spec = ReplicaSpec(positions=np.array([[5.0, 0.5, 0.5]], np.float32),
                       types=np.ones(1, np.int32),
                       box_bound=np.array([[0, 0, 0], [3, 3, 3]], np.float32),
                       epsilon=np.ones((1, 1)), sigma=np.ones((1, 1)), cutoff=1.0, dt=0.001)
    with pytest.raises(ValueError, match="inside box_bound"):
        Engine(spec)


def _nan_at(a, idx):
    import numpy as np

    a = np.array(a, copy=True)
    a[idx] = np.nan
    return a


# One invalid field per case on a 3-chain melt (bonds, angles, dihedrals,
# exclusions, thermostat); each must come back from the C ABI as ValueError
# with the library's message, before any device work (so this runs on CPU).
_ABI_CASES = {
    "positions_nan": (lambda b: dict(positions=_nan_at(b.positions, (0, 0))),
                      "system.positions must be finite"),
    "positions_outside": (lambda b: dict(positions=b.positions + 100.0),
                          "system.positions must be inside box_bound"),
    "velocities_nan": (lambda b: dict(velocities=_nan_at(b.velocities, (1, 2))),
                       "system.velocities must be finite"),
    "box_inverted": (lambda b: dict(box_bound=b.box_bound[::-1].copy()),
                     "upper row must be greater than lower row"),
    "types_zero": (lambda b: dict(types=b.types * 0), "system.types must be dense"),
    "masses_zero": (lambda b: dict(masses=b.masses * 0), "system.masses must be finite and "
                                                         "positive"),
    "tags_duplicate": (lambda b: dict(tags=b.tags * 0 + 1), "permutation of 1..N"),
    "epsilon_negative": (lambda b: dict(epsilon=-b.epsilon),
                         "epsilon and sigma must be finite and positive"),
    "cutoff_zero": (lambda b: dict(cutoff=0.0), "cutoff must be finite and positive"),
    "bond_tag_unknown": (lambda b: dict(bonds=b.bonds[:1] * 0 + [1, 999, 1]),
                         "bonds reference unknown System tags"),
    "bond_type_missing": (lambda b: dict(bonds=b.bonds[:1] * 0 + [1, 2, 2]),
                          "bonds type has no coefficients"),
    "dihedral_d": (lambda b: dict(dihedral_d=[2]), r"dihedral_coeff.d must be \+1 or -1"),
    "dihedral_n": (lambda b: dict(dihedral_n=[-1]), "dihedral_coeff.n must be non-negative"),
    "theta0": (lambda b: dict(angle_theta0=[190.0]), "between 0 and 180 degrees"),
    "exclusion_distance": (lambda b: dict(exclusion_distance=4), "must be 1, 2, or 3"),
    "max_neighbors": (lambda b: dict(max_neighbors=0), "max_neighbors must be positive"),
    "check_every": (lambda b: dict(rebuild_check_every=0),
                    "rebuild_check_every must be positive"),
    "sort_every": (lambda b: dict(sort_every_rebuild=0), "sort_every_rebuild must be positive"),
    "dt_zero": (lambda b: dict(dt=0.0), "dt must be finite and positive"),
    "tau_zero": (lambda b: dict(thermostat=(1.0, 0.0)), "tau must be finite and positive"),
    "temperature_negative": (lambda b: dict(thermostat=(-1.0, 1.0)),
                             "temperature must be finite and non-negative"),
    "units": (lambda b: dict(units="si"), 'units must be "reduced" or "nm_kjmol"'),
}


def _abi_base():
    from beads_b200 import workloads

    return workloads.polymer_melt(n_chains=3, beads=6, seed=1, max_neighbors=64)


@pytest.mark.parametrize("name", sorted(_ABI_CASES))
def test_abi_refuses_invalid_replica(name):
    import dataclasses

    from beads_b200.engine import Engine

    base = _abi_base()
    edit, message = _ABI_CASES[name]
    with pytest.raises(ValueError, match=message):
        Engine(dataclasses.replace(base, **edit(base)))
