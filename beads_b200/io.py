"""Readers for the BEADS binary files written by the engine.

* ``read_beads_trajectory(path)`` (alias ``read_trajectory``): a
  ``BEADS_TRAJECTORY`` v1 file (header: magic, version, endian marker 0x01020304,
  real/index/image/type/tag sizes, units, field mask, particle count, record
  bytes; frames: step u64, box lower[3], upper[3], packed records in the
  writer's slot order).  Join records across frames on ``tag``.
* ``read_state(path)``: a ``BEADS_SNAPSHOT`` v1 final-state file as keyword
  arguments for ``System`` (``System.from_state`` uses it).

The layouts are the reference's file contracts
(native/src/simulation/output/trajectory/trajectory_output.cu:32-45, 555-596;
native/src/simulation/output/snapshot/final_state_output.cu:110-185).
"""

from __future__ import annotations

import os
import struct

import numpy as np

_TRAJ_MAGIC = b"BEADS_TRAJECTORY"
_SNAP_MAGIC = b"BEADS_SNAPSHOT"
_ENDIAN = 0x01020304
_FIELDS = (("tag", 1), ("type", 2), ("position", 4), ("image", 8), ("velocity", 16),
           ("force", 32))


class _Reader:
    def __init__(self, data: bytes, what: str):
        self.data = data
        self.at = 0
        self.what = what

    def take(self, n: int, label: str) -> bytes:
        if self.at + n > len(self.data):
            raise ValueError(f"{self.what} is truncated while reading {label}")
        out = self.data[self.at:self.at + n]
        self.at += n
        return out

    def u32(self, label: str) -> int:
        return struct.unpack("=I", self.take(4, label))[0]

    def u64(self, label: str) -> int:
        return struct.unpack("=Q", self.take(8, label))[0]


def _real_dtype(size: int, what: str):
    if size == 4:
        return np.float32
    if size == 8:
        return np.float64
    raise ValueError(f"{what} real size {size} is not supported; expected 4 or 8")


def read_beads_trajectory(path) -> dict:
    """All frames of a BEADS trajectory (records kept in writer order)."""
    with open(os.fspath(path), "rb") as fh:
        data = fh.read()
    r = _Reader(data, "trajectory")
    if r.take(len(_TRAJ_MAGIC), "magic") != _TRAJ_MAGIC:
        raise ValueError("trajectory magic is not supported")
    version = r.u32("version")
    if version != 1:
        raise ValueError(f"trajectory version {version} is not supported")
    endian = r.u32("endian marker")
    if endian != _ENDIAN:
        raise ValueError("trajectory endian marker is not supported")
    sizes = [r.u32(x) for x in ("real size", "index size", "image size", "type size",
                                "tag size")]
    real = _real_dtype(sizes[0], "trajectory")
    units = r.take(r.u64("units length"), "units").decode("ascii")
    mask = r.u32("field mask")
    n = r.u64("particle count")
    record_bytes = r.u64("record bytes")
    fields = [name for name, bit in _FIELDS if mask & bit]
    rec = []
    for name in fields:
        if name == "tag":
            rec.append(("tag", np.uint32))
        elif name == "type":
            rec.append(("type", np.int32))
        elif name == "image":
            rec.append(("image", np.int32, (3,)))
        else:
            rec.append((name, real, (3,)))
    rec_dtype = np.dtype(rec)
    if rec_dtype.itemsize != record_bytes:
        raise ValueError("trajectory record bytes do not match the field mask")
    frame_dtype = np.dtype([("step", np.uint64), ("box_bound", real, (2, 3)),
                            ("records", rec_dtype, (n,))])
    payload = data[r.at:]
    if len(payload) % frame_dtype.itemsize:
        raise ValueError("Trajectory payload ended before all frames were read.")
    frames = np.frombuffer(payload, dtype=frame_dtype)
    boxes = np.array(frames["box_bound"], copy=True)
    return {
        "version": version, "endian": endian, "real_size": sizes[0], "index_size": sizes[1],
        "image_size": sizes[2], "type_size": sizes[3], "tag_size": sizes[4], "units": units,
        "field_mask": mask, "fields": fields, "n_particles": n, "particle_count": n,
        "record_bytes": record_bytes, "frame_count": int(frames.shape[0]),
        "steps": np.array(frames["step"], copy=True), "box_bounds": boxes,
        "box_lo": boxes[:, 0, :], "box_hi": boxes[:, 1, :],
        "records": np.array(frames["records"], copy=True),
    }


def read_trajectory(path) -> dict:
    """Alias of ``read_beads_trajectory``."""
    return read_beads_trajectory(path)


def read_state(path) -> dict:
    """A final-state snapshot as ``System`` keyword arguments."""
    with open(os.fspath(path), "rb") as fh:
        data = fh.read()
    r = _Reader(data, "state snapshot")
    if r.take(len(_SNAP_MAGIC), "magic") != _SNAP_MAGIC:
        raise ValueError("state snapshot magic is not supported")
    version = r.u32("version")
    if version != 1:
        raise ValueError(f"state snapshot version {version} is not supported")
    real_size, index_size, image_size, type_size, tag_size = (
        r.u32(x) for x in ("real size", "index size", "image size", "type size", "tag size"))
    if r.u32("endian marker") != _ENDIAN:
        raise ValueError("state snapshot endian marker is not supported")
    for label, size in (("index", index_size), ("image", image_size), ("type", type_size),
                        ("tag", tag_size)):
        if size != 4:
            raise ValueError(f"state snapshot {label} size {size} is not supported; expected 4")
    real = _real_dtype(real_size, "state snapshot")
    units = r.take(r.u64("units length"), "units").decode("ascii")
    if units not in ("reduced", "nm_kjmol"):
        raise ValueError(f"state snapshot units {units!r} are not supported")
    r.u64("step")
    n = r.u64("particle count")
    if n <= 0:
        raise ValueError("state snapshot particle count must be positive")

    def arr(dtype, count, label):
        return np.frombuffer(r.take(np.dtype(dtype).itemsize * count, label), dtype=dtype).copy()

    lo, hi = arr(real, 3, "box lower"), arr(real, 3, "box upper")
    tags = arr(np.uint32, n, "tag")
    types = arr(np.int32, n, "type")
    mol = arr(np.uint32, n, "molecule_id")
    mass = arr(real, n, "mass")
    pos = np.stack([arr(real, n, f"position_{c}") for c in "xyz"], axis=1)
    vel = np.stack([arr(real, n, f"velocity_{c}") for c in "xyz"], axis=1)
    img = np.stack([arr(np.int32, n, f"image_{c}") for c in "xyz"], axis=1)
    if r.at != len(data):
        raise ValueError("state snapshot contains trailing bytes")
    return {"units": units, "box_bound": np.stack([lo, hi]), "positions": pos,
            "velocities": vel, "masses": mass, "types": types, "tags": tags,
            "molecule_ids": mol, "images": img}
