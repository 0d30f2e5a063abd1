"""Readers and converters for the files around a BEADS run.

* ``read_beads_trajectory(path)`` (alias ``read_trajectory``): a
  ``BEADS_TRAJECTORY`` v1 file (header: magic, version, endian marker 0x01020304,
  real/index/image/type/tag sizes, units, field mask, particle count, record
  bytes; frames: step u64, box lower[3], upper[3], packed records in the
  writer's slot order).  Join records across frames on ``tag``.
* ``read_state(path)``: a ``BEADS_SNAPSHOT`` v1 final-state file as keyword
  arguments for ``System`` (``System.from_state`` uses it).
* ``read_lammps_data(path, units=...)``: a LAMMPS data file (``Atoms #
  molecular``, optional ``Masses`` / ``Velocities`` / ``Bonds`` / ``Angles`` /
  ``Dihedrals``, orthogonal box) as a ``System``; the reference's importer
  (python/beads/io.py:97-230) accepts and rejects the same inputs.
* ``write_lammps_dump(trajectory_path, dump_path, sort_by_tag=True,
  precision=17)``: a BEADS trajectory as LAMMPS custom dump text
  (python/beads/io.py:278-297, 959-1028).

The layouts are the reference's file contracts
(native/src/simulation/output/trajectory/trajectory_output.cu:32-45, 555-596;
native/src/simulation/output/snapshot/final_state_output.cu:110-185).
"""

from __future__ import annotations

import operator
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


# ---------------------------------------------------------------------------
# LAMMPS data import

_LMP_READ = ("Masses", "Atoms", "Velocities", "Bonds", "Angles", "Dihedrals", "Impropers")
_LMP_UNSUPPORTED = ("Ellipsoids", "Lines", "Triangles", "Bodies")
_LMP_COUNTS = ("atoms", "bonds", "angles", "dihedrals", "impropers", "atom types",
               "bond types", "angle types", "dihedral types", "improper types")
_LMP_TERMS = (("Bonds", "bonds", "bond", 2), ("Angles", "angles", "angle", 3),
              ("Dihedrals", "dihedrals", "dihedral", 4))


def _lmp_section(content: str) -> str | None:
    """The section a keyword line opens (canonical capitalisation), if any."""
    words = " ".join(content.split())
    low = words.lower()
    for name in _LMP_READ + _LMP_UNSUPPORTED:
        if low == name.lower():
            return name
    if low.endswith(" coeffs") or low.endswith(" type labels"):
        return words
    return None


def _lmp_int(tok: str, what: str, minimum: int | None = None) -> int:
    try:
        value = int(tok, 10)
    except ValueError as exc:
        raise ValueError(f"LAMMPS data {what} must be an integer.") from exc
    if minimum == 1 and value <= 0:
        raise ValueError(f"LAMMPS data {what} must be positive.")
    if minimum == 0 and value < 0:
        raise ValueError(f"LAMMPS data {what} must be non-negative.")
    return value


def _lmp_real(tok: str, what: str) -> float:
    try:
        value = float(tok)
    except ValueError as exc:
        raise ValueError(f"LAMMPS data {what} must be numeric.") from exc
    if not np.isfinite(value):
        raise ValueError(f"LAMMPS data {what} must be finite.")
    return value


def _lmp_width(tokens: list[str], width: int, what: str, layout: str = "") -> None:
    if len(tokens) != width:
        suffix = f" ({layout})" if layout else ""
        raise ValueError(f"LAMMPS data {what} expected {width} columns{suffix}, "
                         f"got {len(tokens)}.")


def _lmp_scan(path) -> tuple[dict, dict]:
    """Header values and the (line number, content) rows of every section."""
    header: dict = {}
    sections: dict = {}
    current = None
    with open(os.fspath(path), "r", encoding="utf-8") as fh:
        for number, raw in enumerate(fh, start=1):
            content, hash_, comment = raw.partition("#")
            content = content.strip()
            comment = comment.strip() if hash_ else ""
            if not content:
                continue
            name = _lmp_section(content)
            if name is not None:
                if name in sections:
                    raise ValueError(f"LAMMPS data section {name!r} is duplicated.")
                sections[name] = {"comment": comment, "rows": []}
                current = name
                continue
            if current is not None:
                sections[current]["rows"].append((number, content))
                continue
            tok = content.split()
            bounds = {("xlo", "xhi"): "x", ("ylo", "yhi"): "y", ("zlo", "zhi"): "z"}
            axis = bounds.get(tuple(tok[-2:])) if len(tok) >= 2 else None
            if axis is not None:
                _lmp_width(tok, 4, f"{axis} bounds")
                header[f"{axis}lo"] = _lmp_real(tok[0], f"{axis}lo")
                header[f"{axis}hi"] = _lmp_real(tok[1], f"{axis}hi")
            elif len(tok) >= 3 and tok[-3:] == ["xy", "xz", "yz"]:
                raise ValueError("LAMMPS data import supports only orthogonal box bounds; "
                                 "triclinic tilt factors are unsupported.")
            elif tok[0] in ("avec", "bvec", "cvec") or tok[:2] == ["abc", "origin"]:
                raise ValueError("LAMMPS data import does not support general triclinic boxes.")
            elif len(tok) >= 2 and " ".join(tok[1:]) in _LMP_COUNTS:
                key = " ".join(tok[1:])
                header[key] = _lmp_int(tok[0], key, minimum=0)
            else:
                header.setdefault("title", content)
    return header, sections


def _lmp_dense(what: str, ids) -> None:
    ids = sorted(set(ids))
    if ids and ids != list(range(1, ids[-1] + 1)):
        raise ValueError(f"LAMMPS data {what} type ids must be dense one-based ids without gaps.")


def _lmp_declared(header: dict, key: str, ids, what: str) -> None:
    if key in header and ids:
        top = max(ids)
        if top > header[key]:
            raise ValueError(f"LAMMPS data {what} type id {top} exceeds declared {key} "
                             f"count {header[key]}.")


def read_lammps_data(path, *, units):
    """A LAMMPS data file as a ``System`` (atoms, optional masses and
    velocities, orthogonal bounds, bonds / angles / dihedrals).  Force-field
    coefficient sections are skipped; no unit conversion: ``units`` goes to
    ``System`` as given."""
    from .system import System

    if units is None:
        raise TypeError("read_lammps_data(...) requires the units keyword argument.")
    header, sections = _lmp_scan(path)
    labels = sorted(name for name in sections if name.endswith("Type Labels"))
    if labels:
        raise ValueError(f"LAMMPS data type labels are not supported: {', '.join(labels)}.")
    unsupported = sorted(name for name in sections if name in _LMP_UNSUPPORTED)
    if unsupported:
        raise ValueError("LAMMPS data import does not support sections: "
                         f"{', '.join(unsupported)}.")
    if any(k not in header for k in ("xlo", "xhi", "ylo", "yhi", "zlo", "zhi")):
        raise ValueError("LAMMPS data file is missing required orthogonal box bounds.")
    for axis in "xyz":
        if header[f"{axis}hi"] <= header[f"{axis}lo"]:
            raise ValueError(f"LAMMPS data {axis}hi must be greater than {axis}lo.")
    if "atoms" not in header:
        raise ValueError("LAMMPS data file is missing the atoms count.")
    if "Atoms" not in sections:
        raise ValueError("LAMMPS data file is missing the Atoms section.")
    if header.get("impropers", 0) > 0 or sections.get("Impropers", {"rows": []})["rows"]:
        raise ValueError("LAMMPS data import does not support Impropers. Remove the Impropers "
                         "section before importing the file into BEADS.")

    # Atoms: atom-ID molecule-ID atom-type x y z [ix iy iz]
    style = sections["Atoms"]["comment"]
    if style and style.split()[0].lower() != "molecular":
        raise ValueError("LAMMPS data import supports only Atoms # molecular.")
    atoms = {}
    width = None
    for number, content in sections["Atoms"]["rows"]:
        tok = content.split()
        if len(tok) not in (6, 9):
            raise ValueError(f"LAMMPS data Atoms line {number} must use molecular format: "
                             "atom-ID molecule-ID atom-type x y z [ix iy iz].")
        if width is None:
            width = len(tok)
        elif width != len(tok):
            raise ValueError("LAMMPS data Atoms section must not mix image flags.")
        aid = _lmp_int(tok[0], f"Atoms line {number} atom-ID", minimum=1)
        if aid in atoms:
            raise ValueError(f"LAMMPS data Atoms section duplicates atom ID {aid}.")
        mol = _lmp_int(tok[1], f"Atoms line {number} molecule-ID")
        if mol < 0:
            raise ValueError("LAMMPS data molecule-ID values must be non-negative.")
        atype = _lmp_int(tok[2], f"Atoms line {number} atom-type", minimum=1)
        xyz = [_lmp_real(t, f"Atoms line {number} coordinate") for t in tok[3:6]]
        img = ([_lmp_int(t, f"Atoms line {number} image flag") for t in tok[6:9]]
               if len(tok) == 9 else [0, 0, 0])
        atoms[aid] = (mol, atype, xyz, img)
    n = header["atoms"]
    if len(atoms) != n:
        raise ValueError(f"LAMMPS data atoms count is {n}, but Atoms contains "
                         f"{len(atoms)} rows.")
    if set(atoms) != set(range(1, len(atoms) + 1)):
        raise ValueError("LAMMPS data atom-ID values must satisfy BEADS System.tags: "
                         "a unique 1..N permutation.")
    ids = sorted(atoms)
    mols = [atoms[a][0] for a in ids]
    if any(m <= 0 for m in mols):
        raise ValueError("LAMMPS data molecule-ID values must satisfy BEADS "
                         "System.molecule_ids: positive dense 1-based ids.")
    if set(mols) != set(range(1, len(set(mols)) + 1)) or max(mols, default=0) > len(ids):
        raise ValueError("LAMMPS data molecule-ID values must satisfy BEADS "
                         "System.molecule_ids: positive dense 1-based ids that do not "
                         "exceed the particle count.")
    atypes = [atoms[a][1] for a in ids]
    _lmp_declared(header, "atom types", atypes, "atom")
    _lmp_dense("atom", atypes)

    velocities = None
    if "Velocities" in sections:
        vel = {}
        for number, content in sections["Velocities"]["rows"]:
            tok = content.split()
            _lmp_width(tok, 4, f"Velocities line {number}")
            aid = _lmp_int(tok[0], f"Velocities line {number} atom-ID", minimum=1)
            if aid not in atoms:
                raise ValueError("LAMMPS data Velocities section references unknown atom "
                                 f"ID {aid}.")
            if aid in vel:
                raise ValueError(f"LAMMPS data Velocities section duplicates atom ID {aid}.")
            vel[aid] = [_lmp_real(t, f"Velocities line {number} component") for t in tok[1:4]]
        if set(vel) != set(atoms):
            raise ValueError("LAMMPS data Velocities section must include every atom "
                             "exactly once.")
        velocities = np.array([vel[a] for a in ids], np.float64)

    masses = None
    if "Masses" in sections:
        per_type = {}
        for number, content in sections["Masses"]["rows"]:
            tok = content.split()
            _lmp_width(tok, 2, f"Masses line {number}", "atom-type mass")
            t = _lmp_int(tok[0], f"Masses line {number} atom type", minimum=1)
            if t in per_type:
                raise ValueError(f"LAMMPS data Masses section duplicates atom type {t}.")
            m = _lmp_real(tok[1], f"Masses line {number} mass")
            if m <= 0.0:
                raise ValueError("LAMMPS data masses must be positive.")
            per_type[t] = m
        _lmp_declared(header, "atom types", list(per_type), "Masses atom")
        missing = sorted(set(atypes) - set(per_type))
        if missing:
            raise ValueError("LAMMPS data Masses section is missing atom types: "
                             f"{', '.join(str(t) for t in missing)}.")
        masses = np.array([per_type[t] for t in atypes], np.float64)

    # Bonds / Angles / Dihedrals: id type atom1 .. atomK  ->  (atom1 .. atomK, type)
    terms = {}
    for section, count_key, what, k in _LMP_TERMS:
        rows = []
        seen = set()
        layout = "id type " + " ".join(f"atom{q + 1}" for q in range(k))
        for number, content in sections.get(section, {"rows": []})["rows"]:
            tok = content.split()
            _lmp_width(tok, k + 2, f"{section} line {number}", layout)
            tid = _lmp_int(tok[0], f"{section} line {number} id", minimum=1)
            if tid in seen:
                raise ValueError(f"LAMMPS data {section} section duplicates id {tid}.")
            seen.add(tid)
            ttype = _lmp_int(tok[1], f"{section} line {number} type", minimum=1)
            refs = [_lmp_int(t, f"{section} line {number} atom id", minimum=1)
                    for t in tok[2:2 + k]]
            for aid in refs:
                if aid not in atoms:
                    raise ValueError(f"LAMMPS data {section} section references unknown "
                                     f"atom ID {aid}.")
            rows.append((*refs, ttype))
        terms[count_key] = rows
    for _, count_key, _, _ in _LMP_TERMS:
        if count_key in header and header[count_key] != len(terms[count_key]):
            raise ValueError(f"LAMMPS data {count_key} count is {header[count_key]}, but the "
                             f"section contains {len(terms[count_key])} rows.")
    for _, count_key, what, _ in _LMP_TERMS:
        types = [row[-1] for row in terms[count_key]]
        _lmp_declared(header, f"{what} types", types, what)
    for _, count_key, what, _ in _LMP_TERMS:
        _lmp_dense(f"{what} topology", [row[-1] for row in terms[count_key]])

    system = System(
        box_bound=np.array([[header["xlo"], header["ylo"], header["zlo"]],
                            [header["xhi"], header["yhi"], header["zhi"]]], np.float64),
        positions=np.array([atoms[a][2] for a in ids], np.float64),
        types=np.array(atypes, np.int64), velocities=velocities, masses=masses,
        tags=np.array(ids, np.uint64), molecule_ids=np.array(mols, np.uint64),
        images=np.array([atoms[a][3] for a in ids], np.int64), units=units)
    if any(terms.values()):
        system.set_topology(bonds=terms["bonds"], angles=terms["angles"],
                            dihedrals=terms["dihedrals"])
    return system


# ---------------------------------------------------------------------------
# LAMMPS dump export

def write_lammps_dump(trajectory_path, dump_path, *, sort_by_tag: bool = True,
                      precision: int = 17) -> None:
    """A BEADS trajectory as LAMMPS custom dump text: one ``ITEM: TIMESTEP``
    block per frame, periodic bounds, columns id [type] [x y z] [ix iy iz]
    [vx vy vz] [fx fy fz] as the trajectory holds them, rows in tag order (or
    the writer's slot order with ``sort_by_tag=False``), reals printed with
    ``precision`` significant digits (1-17)."""
    if not isinstance(sort_by_tag, bool):
        raise TypeError("write_lammps_dump(...) sort_by_tag must be a bool.")
    if isinstance(precision, (bool, np.bool_)):
        raise TypeError("write_lammps_dump(...) precision must be an integer, not bool.")
    try:
        precision = int(operator.index(precision))
    except TypeError as exc:
        raise TypeError("write_lammps_dump(...) precision must be an integer.") from exc
    if not 1 <= precision <= 17:
        raise ValueError("write_lammps_dump(...) precision must be between 1 and 17.")
    traj = read_beads_trajectory(trajectory_path)
    fields = traj["fields"]
    if "tag" not in fields:
        raise ValueError("write_lammps_dump(...) needs a trajectory with the tag field.")
    columns = ["id"]
    for name, cols in (("type", ["type"]), ("position", ["x", "y", "z"]),
                       ("image", ["ix", "iy", "iz"]), ("velocity", ["vx", "vy", "vz"]),
                       ("force", ["fx", "fy", "fz"])):
        if name in fields:
            columns += cols

    def real(x) -> str:
        return f"{float(x):.{precision}g}"

    n = int(traj["n_particles"])
    with open(os.fspath(dump_path), "w", encoding="utf-8") as out:
        for f in range(traj["frame_count"]):
            rec = traj["records"][f]
            order = np.argsort(rec["tag"], kind="stable") if sort_by_tag else np.arange(n)
            box = traj["box_bounds"][f]
            out.write(f"ITEM: TIMESTEP\n{int(traj['steps'][f])}\n")
            out.write(f"ITEM: NUMBER OF ATOMS\n{n}\n")
            out.write("ITEM: BOX BOUNDS pp pp pp\n")
            for axis in range(3):
                out.write(f"{real(box[0, axis])} {real(box[1, axis])}\n")
            out.write(f"ITEM: ATOMS {' '.join(columns)}\n")
            for k in order:
                row = rec[k]
                vals = [str(int(row["tag"]))]
                if "type" in fields:
                    vals.append(str(int(row["type"])))
                if "position" in fields:
                    vals += [real(c) for c in row["position"]]
                if "image" in fields:
                    vals += [str(int(c)) for c in row["image"]]
                if "velocity" in fields:
                    vals += [real(c) for c in row["velocity"]]
                if "force" in fields:
                    vals += [real(c) for c in row["force"]]
                out.write(" ".join(vals) + "\n")
