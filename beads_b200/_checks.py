"""Input checks shared by the builder objects.

The dtypes are the engine's (``build_info()``): float32 reals, int32 types and
images, uint32 tags / indices, uint64 run steps.  Error types follow the
reference's Python layer (python/beads/_validation.py, _params.py): TypeError
for a wrong kind of value, ValueError for a wrong value.
"""

from __future__ import annotations

from types import MappingProxyType
from typing import Any, Mapping

import numpy as np

REAL = np.dtype(np.float32)
TYPE = np.dtype(np.int32)
INDEX = np.dtype(np.uint32)
IMAGE = np.dtype(np.int32)
RUNSTEP = np.dtype(np.uint64)

_INT64 = np.iinfo(np.int64)


def _is_bool(value) -> bool:
    return isinstance(value, (bool, np.bool_))


def _is_int(value) -> bool:
    return isinstance(value, (int, np.integer)) and not _is_bool(value)


def real_array(name: str, value, shape=None) -> np.ndarray:
    probe = np.asarray(value)
    if probe.dtype.kind in "bOSUc":
        raise TypeError(f"{name} must contain real numeric values")
    out = np.array(value, dtype=REAL, copy=True, order="C")
    if shape is not None and out.shape != tuple(shape):
        raise ValueError(f"{name} must have shape {tuple(shape)}")
    if not np.all(np.isfinite(out)):
        raise ValueError(f"{name} must be finite")
    return out


def rows3(name: str, value, n_rows=None) -> np.ndarray:
    out = real_array(name, value)
    if out.ndim != 2 or out.shape[1] != 3:
        raise ValueError(f"{name} must have shape (n_particles, 3)")
    if n_rows is not None and out.shape[0] != n_rows:
        raise ValueError(f"{name} must have one row per particle")
    return out


def int_array(name: str, value, shape=None, dtype=TYPE) -> np.ndarray:
    probe = np.asarray(value)
    if probe.dtype.kind in "bOSUfc":
        raise TypeError(f"{name} must contain integer values")
    if shape is not None and probe.shape != tuple(shape):
        raise ValueError(f"{name} must have shape {tuple(shape)}")
    limits = np.iinfo(dtype)
    if probe.size and (int(probe.min()) < limits.min or int(probe.max()) > limits.max):
        raise ValueError(
            f"{name} contains values outside the supported {np.dtype(dtype).name} range")
    return np.array(value, dtype=dtype, copy=True, order="C")


def positive_int(name: str, value) -> int:
    if not _is_int(value):
        raise TypeError(f"{name} must be an integer")
    if value <= 0:
        raise ValueError(f"{name} must be positive")
    return int(value)


def positive_index(name: str, value) -> int:
    out = positive_int(name, value)
    if out > np.iinfo(INDEX).max:
        raise ValueError(f"{name} contains values outside the supported uint32 range")
    return out


def positive_type(name: str, value) -> int:
    out = positive_int(name, value)
    if out > np.iinfo(TYPE).max:
        raise ValueError(f"{name} contains values outside the supported int32 range")
    return out


def nonnegative_steps(name: str, value) -> int:
    if not _is_int(value):
        raise TypeError(f"{name} must be an integer")
    out = int(value)
    if out < 0:
        raise ValueError(f"{name} must be non-negative")
    if out > np.iinfo(RUNSTEP).max:
        raise ValueError(f"{name} contains values outside the supported uint64 range")
    return out


def positive_steps(name: str, value) -> int:
    out = nonnegative_steps(name, value)
    if out == 0:
        raise ValueError(f"{name} must be positive")
    return out


def nonnegative_real(name: str, value) -> float:
    if _is_bool(value) or not isinstance(value, (int, float, np.integer, np.floating)):
        raise TypeError(f"{name} must be a real number")
    out = float(value)
    if not np.isfinite(out):
        raise ValueError(f"{name} must be finite")
    if out < 0.0:
        raise ValueError(f"{name} must be non-negative")
    return out


def scalar_params(context: str, params: Mapping[str, object], *, allow_bool: bool) -> dict:
    """Freeze a keyword-parameter mapping to plain Python scalars."""
    out: dict[str, Any] = {}
    for key, value in params.items():
        if not isinstance(key, str) or not key:
            raise TypeError(f"{context} names must be non-empty strings.")
        if _is_bool(value):
            if not allow_bool:
                raise TypeError(f"{context} {key} must not be bool.")
            out[key] = bool(value)
        elif _is_int(value):
            if not (_INT64.min <= int(value) <= _INT64.max):
                raise ValueError(
                    f"{context} {key} contains values outside the supported int64 range.")
            out[key] = int(value)
        elif isinstance(value, (float, np.floating)):
            f = float(value)
            if not np.isfinite(f):
                raise ValueError(f"{context} {key} must be finite.")
            with np.errstate(over="ignore"):
                if not np.isfinite(np.float32(f)):
                    raise ValueError(f"{context} {key} must be representable as float32.")
            out[key] = f
        elif isinstance(value, str):
            out[key] = value
        else:
            kinds = "bool, int, float, or string" if allow_bool else "int, float, or string"
            raise TypeError(f"{context} {key} must be {kinds}.")
    return out


def frozen(mapping: Mapping[str, Any]) -> Mapping[str, Any]:
    return MappingProxyType(dict(mapping))
