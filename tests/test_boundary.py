"""The C-ABI library loads and exports every entry point include/beads_b200.h
declares (no compute call: this runs without a GPU)."""

from __future__ import annotations

import ctypes
import re

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
    import pytest

    from beads_b200.engine import Engine, ReplicaSpec

    spec = ReplicaSpec(positions=np.array([[5.0, 0.5, 0.5]], np.float32),
                       types=np.ones(1, np.int32),
                       box_bound=np.array([[0, 0, 0], [3, 3, 3]], np.float32),
                       epsilon=np.ones((1, 1)), sigma=np.ones((1, 1)), cutoff=1.0, dt=0.001)
    with pytest.raises(ValueError, match="inside box_bound"):
        Engine(spec)
