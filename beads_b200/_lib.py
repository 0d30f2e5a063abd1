"""ctypes binding of ``libbeads_b200.so`` (the C ABI in include/beads_b200.h).

The library is built in-tree (``python -m beads_b200.build``).  Loading fails
loudly when it is missing: there is no fallback implementation.
"""

from __future__ import annotations

import ctypes
import json
import pathlib

import numpy as np

PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG / "libbeads_b200.so"

OK = 0
ERR_INVALID = -1
ERR_RUNTIME = -2
ERR_OVERFLOW = -3
ERR_CUDA = -4
ERR_NEIGHBOR_OVERFLOW = -5
ERR_NONFINITE = -6
ERR_INTERRUPTED = -7

UNITS = {"reduced": 0, "nm_kjmol": 1}
FIELD_BITS = {"tag": 1, "type": 2, "position": 4, "image": 8, "velocity": 16, "force": 32}
ECHO = {"none": 0, "screen": 1, "log": 2, "both": 3}

c_f32p = ctypes.POINTER(ctypes.c_float)
c_f64p = ctypes.POINTER(ctypes.c_double)
c_u32p = ctypes.POINTER(ctypes.c_uint32)
c_i32p = ctypes.POINTER(ctypes.c_int32)


class SystemDesc(ctypes.Structure):
    _fields_ = [
        ("n_particles", ctypes.c_uint32),
        ("units", ctypes.c_int32),
        ("box_lo", ctypes.c_float * 3),
        ("box_hi", ctypes.c_float * 3),
        ("positions", c_f32p),
        ("velocities", c_f32p),
        ("masses", c_f32p),
        ("types", c_i32p),
        ("tags", c_u32p),
        ("molecule_ids", c_u32p),
        ("images", c_i32p),
        ("n_bonds", ctypes.c_uint32),
        ("bonds", c_u32p),
        ("n_angles", ctypes.c_uint32),
        ("angles", c_u32p),
        ("n_dihedrals", ctypes.c_uint32),
        ("dihedrals", c_u32p),
    ]


class ForceFieldDesc(ctypes.Structure):
    _fields_ = [
        ("n_types", ctypes.c_int32),
        ("lj_epsilon", c_f64p),
        ("lj_sigma", c_f64p),
        ("lj_cutoff", ctypes.c_double),
        ("lj_shift", ctypes.c_int32),
        ("n_bond_types", ctypes.c_int32),
        ("bond_k", c_f64p),
        ("bond_r0", c_f64p),
        ("n_angle_types", ctypes.c_int32),
        ("angle_k", c_f64p),
        ("angle_theta0_deg", c_f64p),
        ("n_dihedral_types", ctypes.c_int32),
        ("dihedral_k", c_f64p),
        ("dihedral_d", c_i32p),
        ("dihedral_n", c_i32p),
        ("exclusion_distance", ctypes.c_int32),
    ]


class NeighborDesc(ctypes.Structure):
    _fields_ = [
        ("cutoff_buffer", ctypes.c_double),
        ("rebuild_check_every", ctypes.c_uint64),
        ("sort_every_rebuild", ctypes.c_uint64),
        ("max_neighbors", ctypes.c_uint32),
    ]


class DynamicsDesc(ctypes.Structure):
    _fields_ = [
        ("dt", ctypes.c_double),
        ("thermostat", ctypes.c_int32),
        ("temperature", ctypes.c_double),
        ("tau", ctypes.c_double),
    ]


class Observables(ctypes.Structure):
    _fields_ = [
        ("step", ctypes.c_uint64),
        ("pair_pe", ctypes.c_double),
        ("bond_pe", ctypes.c_double),
        ("angle_pe", ctypes.c_double),
        ("dihedral_pe", ctypes.c_double),
        ("pe", ctypes.c_double),
        ("ke", ctypes.c_double),
        ("virial", ctypes.c_double),
        ("temp", ctypes.c_double),
        ("press", ctypes.c_double),
        ("neighbor_build_count", ctypes.c_uint64),
        ("dangerous_rebuild_count", ctypes.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


INTERRUPT_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p)


class RunDesc(ctypes.Structure):
    _fields_ = [
        ("system", ctypes.POINTER(SystemDesc)),
        ("forcefield", ctypes.POINTER(ForceFieldDesc)),
        ("neighbor", ctypes.POINTER(NeighborDesc)),
        ("dynamics", ctypes.POINTER(DynamicsDesc)),
        ("runsteps", ctypes.c_uint64),
        ("thermo_every", ctypes.c_uint64),
        ("thermo_prefix", ctypes.c_char_p),
        ("trajectory_every", ctypes.c_uint64),
        ("trajectory_prefix", ctypes.c_char_p),
        ("trajectory_fields", ctypes.c_uint32),
        ("final_state_prefix", ctypes.c_char_p),
        ("log_echo", ctypes.c_int32),
        ("log_prefix", ctypes.c_char_p),
        ("thermostat_name", ctypes.c_char_p),
        ("exclusion_policy", ctypes.c_char_p),
        ("interrupt", INTERRUPT_FN),
        ("interrupt_user", ctypes.c_void_p),
    ]


EXPORTED = (
    "beads_build_info",
    "beads_last_error",
    "beads_execute",
    "beads_ctx_create",
    "beads_batch_create",
    "beads_ctx_destroy",
    "beads_eval",
    "beads_run",
    "beads_get_state",
    "beads_set_state",
    "beads_upload_all",
    "beads_download_all",
    "beads_ctx_info",
    "beads_minimize",
    "beads_profile",
    "beads_list_stats",
    "beads_counters",
    "beads_launch_counts",
    "beads_set_tuning",
    "beads_get_tuning",
    "beads_set_list_layout",
    "beads_get_list_layout",
    "beads_set_lj",
    "beads_adjoint_forward",
    "beads_adjoint_backward",
    "beads_set_bonded",
    "beads_adjoint_bonded_grads",
    "beads_cell_sort_static",
    "beads_debug_cells",
    "beads_debug_neighbors",
    "beads_debug_plan",
)

_lib = None


def load():
    """Load the in-tree shared library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            "BEADS native extension is not built: "
            f"{LIB_PATH} is missing (run `python -m beads_b200.build`)."
        )
    L = ctypes.CDLL(str(LIB_PATH))
    vp = ctypes.c_void_p
    L.beads_build_info.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    L.beads_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    L.beads_execute.argtypes = [ctypes.POINTER(RunDesc)]
    L.beads_ctx_create.argtypes = [ctypes.POINTER(SystemDesc), ctypes.POINTER(ForceFieldDesc),
                                   ctypes.POINTER(NeighborDesc), ctypes.POINTER(DynamicsDesc),
                                   ctypes.POINTER(vp)]
    L.beads_batch_create.argtypes = [ctypes.c_uint32, ctypes.POINTER(SystemDesc),
                                     ctypes.POINTER(ForceFieldDesc), ctypes.POINTER(NeighborDesc),
                                     ctypes.POINTER(DynamicsDesc), ctypes.POINTER(vp)]
    L.beads_ctx_destroy.argtypes = [vp]
    L.beads_ctx_destroy.restype = None
    L.beads_eval.argtypes = [vp, ctypes.POINTER(Observables)]
    L.beads_run.argtypes = [vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(Observables)]
    L.beads_get_state.argtypes = [vp, ctypes.c_uint32, vp, vp, vp, vp]
    L.beads_set_state.argtypes = [vp, ctypes.c_uint32, vp, vp]
    L.beads_upload_all.argtypes = [vp, vp, vp]
    L.beads_download_all.argtypes = [vp, vp, vp]
    L.beads_ctx_info.argtypes = [vp, ctypes.POINTER(ctypes.c_uint32),
                                 ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(vp)]
    L.beads_minimize.argtypes = [vp, ctypes.c_uint32, ctypes.c_float, ctypes.c_float]
    L.beads_profile.argtypes = [vp, ctypes.c_int32, ctypes.c_uint32, ctypes.POINTER(ctypes.c_double)]
    L.beads_list_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint32)]
    L.beads_counters.argtypes = [vp, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint64)]
    L.beads_launch_counts.argtypes = [vp, ctypes.POINTER(ctypes.c_uint32),
                                      ctypes.POINTER(ctypes.c_uint32)]
    L.beads_set_tuning.argtypes = [vp, ctypes.POINTER(ctypes.c_int32)]
    L.beads_get_tuning.argtypes = [vp, ctypes.POINTER(ctypes.c_int32)]
    L.beads_set_list_layout.argtypes = [vp, ctypes.c_int32]
    L.beads_get_list_layout.argtypes = [vp, ctypes.POINTER(ctypes.c_int32)]
    L.beads_set_lj.argtypes = [vp, ctypes.c_uint32, vp, vp]
    L.beads_adjoint_forward.argtypes = [vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, vp]
    L.beads_adjoint_backward.argtypes = [vp, vp, vp, vp, vp, vp]
    L.beads_set_bonded.argtypes = [vp, ctypes.c_uint32, vp, vp, vp, vp, vp]
    L.beads_adjoint_bonded_grads.argtypes = [vp, vp, vp, vp]
    L.beads_cell_sort_static.argtypes = [vp, ctypes.c_uint32, ctypes.POINTER(ctypes.c_float),
                                         ctypes.POINTER(ctypes.c_float), ctypes.c_double,
                                         ctypes.c_double, vp, vp, vp, ctypes.c_uint32,
                                         ctypes.POINTER(ctypes.c_uint32), vp]
    L.beads_debug_cells.argtypes = [vp, ctypes.c_uint32, vp]
    L.beads_debug_neighbors.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, vp, vp]
    L.beads_debug_plan.argtypes = [vp, ctypes.c_uint32, ctypes.POINTER(ctypes.c_int32), vp]
    for name in EXPORTED:
        if name != "beads_ctx_destroy":
            getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def last_error() -> str:
    buf = ctypes.create_string_buffer(4096)
    load().beads_last_error(buf, len(buf))
    return buf.value.decode("utf-8", "replace")


def check(status: int) -> None:
    """Raise the Python exception the reference raises for this status."""
    if status == OK:
        return
    message = last_error()
    if status == ERR_INVALID:
        raise ValueError(message)
    if status == ERR_OVERFLOW:
        raise OverflowError(message)
    if status == ERR_INTERRUPTED:
        raise KeyboardInterrupt(message)
    raise RuntimeError(message)


def build_info() -> dict:
    buf = ctypes.create_string_buffer(512)
    check(load().beads_build_info(buf, len(buf)))
    return json.loads(buf.value.decode())


def _as(arr, dtype, ctype):
    return np.ascontiguousarray(arr, dtype=dtype), ctypes.POINTER(ctype)


class Keep:
    """Holds the NumPy buffers a descriptor points into."""

    def __init__(self) -> None:
        self.items: list = []

    def ptr(self, arr, dtype, ctype):
        if arr is None:
            return ctypes.POINTER(ctype)()
        a = np.ascontiguousarray(arr, dtype=dtype)
        self.items.append(a)
        return a.ctypes.data_as(ctypes.POINTER(ctype))
