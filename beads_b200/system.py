"""``System``: particles, box, units and topology (the reference's
python/beads/_system.py and _topology.py contract)."""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _checks as C


@dataclass(frozen=True)
class Topology:
    bonds: tuple[tuple[int, int, int], ...] = ()
    angles: tuple[tuple[int, int, int, int], ...] = ()
    dihedrals: tuple[tuple[int, int, int, int, int], ...] = ()


def _records(name: str, records, width: int) -> list[tuple]:
    if records is None:
        return []
    if isinstance(records, (str, bytes)):
        raise TypeError(f"{name} must be an iterable of topology records")
    try:
        items = list(records)
    except TypeError as exc:
        raise TypeError(f"{name} must be an iterable of topology records") from exc
    out = []
    for k, rec in enumerate(items):
        if isinstance(rec, (str, bytes)):
            raise TypeError(f"{name}[{k}] must be a topology record")
        try:
            values = tuple(rec)
        except TypeError as exc:
            raise TypeError(f"{name}[{k}] must be a topology record") from exc
        if len(values) != width:
            raise ValueError(f"{name}[{k}] must contain exactly {width} values")
        out.append(values)
    return out


def _tag(name: str, k: int, m: int, value, tags: frozenset) -> int:
    t = C.positive_index(f"{name}[{k}][{m}]", value)
    if t not in tags:
        raise ValueError(f"{name}[{k}] references unknown System tag {t}")
    return t


def _dense_types(label: str, types) -> None:
    seen = sorted(set(types))
    if seen and seen != list(range(1, len(seen) + 1)):
        raise ValueError(f"{label} topology types must be dense one-based ids without gaps")


def build_topology(bonds, angles, dihedrals, tags) -> Topology:
    """Canonical topology: bonds (i < j), angles (i < k around j), dihedrals
    (lexicographically smaller of the two directions); duplicates rejected;
    angles and dihedrals must run along bonds."""
    tagset = frozenset(int(t) for t in tags)
    canon_b, seen = [], set()
    for k, rec in enumerate(_records("bonds", bonds, 3)):
        i = _tag("bonds", k, 0, rec[0], tagset)
        j = _tag("bonds", k, 1, rec[1], tagset)
        ty = C.positive_type(f"bonds[{k}] type", rec[2])
        if i == j:
            raise ValueError("bonds entries must reference distinct tags")
        i, j = min(i, j), max(i, j)
        if (i, j) in seen:
            raise ValueError("bonds must not contain duplicate records")
        seen.add((i, j))
        canon_b.append((i, j, ty))
    _dense_types("bond", [b[2] for b in canon_b])
    pairs = {(b[0], b[1]) for b in canon_b}

    def bonded(a, b):
        return (min(a, b), max(a, b)) in pairs

    canon_a, seen = [], set()
    for k, rec in enumerate(_records("angles", angles, 4)):
        i, j, m = (_tag("angles", k, q, rec[q], tagset) for q in range(3))
        ty = C.positive_type(f"angles[{k}] type", rec[3])
        if len({i, j, m}) != 3:
            raise ValueError("angles entries must reference three distinct tags")
        if m < i:
            i, m = m, i
        if (i, j, m) in seen:
            raise ValueError("angles must not contain duplicate records")
        seen.add((i, j, m))
        canon_a.append((i, j, m, ty))
    _dense_types("angle", [a[3] for a in canon_a])
    for i, j, m, _ in canon_a:
        if not (bonded(i, j) and bonded(j, m)):
            raise ValueError("angles require supporting topology bonds for each edge")

    canon_d, seen = [], set()
    for k, rec in enumerate(_records("dihedrals", dihedrals, 5)):
        quad = tuple(_tag("dihedrals", k, q, rec[q], tagset) for q in range(4))
        ty = C.positive_type(f"dihedrals[{k}] type", rec[4])
        if len(set(quad)) != 4:
            raise ValueError("dihedrals entries must reference four distinct tags")
        quad = min(quad, quad[::-1])
        if quad in seen:
            raise ValueError("dihedrals must not contain duplicate records")
        seen.add(quad)
        canon_d.append((*quad, ty))
    _dense_types("dihedral", [d[4] for d in canon_d])
    for a, b, c, d, _ in canon_d:
        if not (bonded(a, b) and bonded(b, c) and bonded(c, d)):
            raise ValueError("dihedrals require supporting topology bonds for each edge")
    return Topology(tuple(canon_b), tuple(canon_a), tuple(canon_d))


def _permutation(name: str, values, n: int) -> np.ndarray:
    arr = C.int_array(name, values, (n,), dtype=C.INDEX)
    if not np.array_equal(np.sort(arr), np.arange(1, n + 1, dtype=C.INDEX)):
        raise ValueError(f"{name} must be a permutation of 1..N")
    return arr


def _dense_ids(name: str, values, n: int) -> np.ndarray:
    arr = C.int_array(name, values, (n,), dtype=C.INDEX)
    if arr.size == 0 or np.any(arr < 1):
        raise ValueError(f"{name} must be one-based positive integers")
    u = np.unique(arr)
    if int(u[-1]) > n or not np.array_equal(u, np.arange(1, u.size + 1)):
        raise ValueError(f"{name} must form a contiguous 1-based set starting at 1")
    return arr


def _dense_types_array(values, n: int) -> np.ndarray:
    arr = C.int_array("types", values, (n,), dtype=C.TYPE)
    if arr.size == 0 or np.any(arr < 1):
        raise ValueError("types must be one-based positive integers")
    u = np.unique(arr)
    if not np.array_equal(u, np.arange(1, u.size + 1)):
        raise ValueError("types must be dense one-based ids without gaps")
    return arr


class System:
    """Particles in an orthorhombic periodic box.

    Required keywords: ``positions`` (N x 3, inside ``[lower, upper)``),
    ``types`` (dense 1-based), ``box_bound`` (2 x 3: lower row, upper row),
    ``units`` ("reduced" or "nm_kjmol").  Optional: ``velocities`` (zeros),
    ``masses`` (ones), ``tags`` (1..N), ``molecule_ids`` (ones), ``images``
    (zeros).  Frozen once bound to a ``Simulation``.
    """

    def __init__(self, *, positions, types, box_bound=None, velocities=None, masses=None,
                 tags=None, molecule_ids=None, images=None, units=None):
        if units is None:
            raise TypeError('System requires explicit units="reduced" or units="nm_kjmol".')
        if not isinstance(units, str):
            raise TypeError("units must be a string")
        if units not in ("reduced", "nm_kjmol"):
            raise ValueError('units must be "reduced" or "nm_kjmol"')
        pos = C.real_array("positions", positions)
        if pos.ndim != 2 or pos.shape[1] != 3:
            if pos.ndim == 1 and pos.shape[0] == 0:
                raise ValueError("positions must contain at least one particle")
            raise ValueError("positions must have shape (n_particles, 3)")
        n = pos.shape[0]
        if n == 0:
            raise ValueError("positions must contain at least one particle")
        if box_bound is None:
            raise TypeError("System requires box_bound=")
        box = C.real_array("box_bound", box_bound, (2, 3))
        if np.any(box[1] - box[0] <= 0.0):
            raise ValueError("box_bound upper row must be greater than lower row")
        if np.any(pos < box[0]) or np.any(pos >= box[1]):
            raise ValueError("positions must be inside box_bound")
        vel = np.zeros_like(pos) if velocities is None else C.rows3("velocities", velocities, n)
        mass = (np.ones(n, C.REAL) if masses is None
                else C.real_array("masses", masses, (n,)))
        if np.any(mass <= 0.0):
            raise ValueError("masses must be finite and positive")
        self._positions = pos
        self._box_bound = box
        self._types = _dense_types_array(types, n)
        self._velocities = vel
        self._masses = mass
        self._tags = (np.arange(1, n + 1, dtype=C.INDEX) if tags is None
                      else _permutation("tags", tags, n))
        self._molecule_ids = (np.ones(n, C.INDEX) if molecule_ids is None
                              else _dense_ids("molecule_ids", molecule_ids, n))
        self._images = (np.zeros((n, 3), C.IMAGE) if images is None
                        else C.int_array("images", images, (n, 3), dtype=C.IMAGE))
        self._units = units
        self._topology = Topology()
        self._frozen = False

    # read-only views (arrays become non-writable once frozen)
    positions = property(lambda self: self._positions)
    box_bound = property(lambda self: self._box_bound)
    types = property(lambda self: self._types)
    velocities = property(lambda self: self._velocities)
    masses = property(lambda self: self._masses)
    tags = property(lambda self: self._tags)
    molecule_ids = property(lambda self: self._molecule_ids)
    images = property(lambda self: self._images)
    units = property(lambda self: self._units)
    topology = property(lambda self: self._topology)

    @property
    def n_particles(self) -> int:
        return int(self._positions.shape[0])

    @classmethod
    def from_state(cls, path) -> "System":
        from .io import read_state

        return cls(**read_state(path))

    def set_topology(self, *, bonds=None, angles=None, dihedrals=None) -> "System":
        if self._frozen:
            raise RuntimeError("System is frozen after binding to a Simulation.")
        self._topology = build_topology(bonds, angles, dihedrals, self._tags.tolist())
        return self

    def _freeze(self) -> "System":
        for name in ("_positions", "_box_bound", "_types", "_velocities", "_masses", "_tags",
                     "_molecule_ids", "_images"):
            arr = np.array(getattr(self, name), copy=True, order="C")
            arr.setflags(write=False)
            setattr(self, name, arr)
        self._frozen = True
        return self
