"""Generates tests/golden/lammps/: LAMMPS data files, what the reference's
own ``beads.io.read_lammps_data`` made of them (arrays, topology, or the
exception it raised), a small BEADS trajectory and the reference's
``beads.io.write_lammps_dump`` text for it.

Needs the reference checkout (its pure-Python package is imported from
<reference>/python; nothing native runs):

    python tests/golden/make_lammps_fixtures.py <reference checkout>
"""

from __future__ import annotations

import json
import pathlib
import struct
import sys

import numpy as np

OUT = pathlib.Path(__file__).resolve().parent / "lammps"

CHAIN = """LAMMPS data file: two short chains  # title

6 atoms
3 atom types
4 bonds
1 bond types
2 angles
1 angle types
1 dihedrals
1 dihedral types

0.0 10.0 xlo xhi
-5.0 5.0 ylo yhi
0.0 8.0 zlo zhi

Masses

1 1.0
2 2.5   # heavier bead
3 0.75

Pair Coeffs # lj/cut

1 1.0 1.0
2 1.0 1.0
3 1.0 1.0

Atoms # molecular

3 1 2 3.0 0.5 1.0 0 1 -1
1 1 1 1.0 0.5 1.0 0 0 0
2 1 1 2.0 0.5 1.0 0 0 0
4 1 3 4.0 0.5 1.0 1 0 0
6 2 2 7.5 -2.0 6.0 0 0 2
5 2 1 6.5 -2.0 6.0 0 0 2

Velocities

1 0.1 0.0 0.0
2 0.0 0.2 0.0
3 0.0 0.0 0.3
4 -0.1 0.0 0.0
5 0.0 -0.2 0.0
6 0.0 0.0 -0.3

Bonds

1 1 1 2
2 1 2 3
3 1 3 4
4 1 5 6

Angles

1 1 1 2 3
2 1 2 3 4

Dihedrals

1 1 1 2 3 4
"""

PLAIN = """four beads in a unit box

4 atoms
2 atom types
0 1 xlo xhi
0 1 ylo yhi
0 1 zlo zhi

Atoms

2 1 2 0.25 0.25 0.25
1 1 1 0.75 0.75 0.75
4 2 2 0.25 0.75 0.25
3 2 1 0.75 0.25 0.75
"""


def _replace(text: str, old: str, new: str) -> str:
    assert old in text, old
    return text.replace(old, new, 1)


INVALID = {
    "no_bounds": _replace(PLAIN, "0 1 zlo zhi\n", ""),
    "inverted_bounds": _replace(PLAIN, "0 1 ylo yhi", "1 0 ylo yhi"),
    "triclinic": _replace(PLAIN, "0 1 zlo zhi\n", "0 1 zlo zhi\n0.1 0 0 xy xz yz\n"),
    "no_atoms_count": _replace(PLAIN, "4 atoms\n", ""),
    "atoms_count_mismatch": _replace(PLAIN, "4 atoms", "5 atoms"),
    "atomic_style": _replace(PLAIN, "Atoms\n", "Atoms # atomic\n"),
    "bad_width": _replace(PLAIN, "2 1 2 0.25 0.25 0.25", "2 1 2 0.25 0.25"),
    "mixed_images": _replace(PLAIN, "2 1 2 0.25 0.25 0.25", "2 1 2 0.25 0.25 0.25 0 0 0"),
    "duplicate_id": _replace(PLAIN, "4 2 2 0.25 0.75 0.25", "2 2 2 0.25 0.75 0.25"),
    "ids_not_permutation": _replace(PLAIN, "4 2 2 0.25 0.75 0.25", "7 2 2 0.25 0.75 0.25"),
    "molecule_zero": _replace(PLAIN, "4 2 2 0.25 0.75 0.25", "4 0 2 0.25 0.75 0.25"),
    "molecule_gap": _replace(_replace(PLAIN, "4 2 2 0.25 0.75 0.25", "4 3 2 0.25 0.75 0.25"),
                             "3 2 1 0.75 0.25 0.75", "3 3 1 0.75 0.25 0.75"),
    "type_gap": _replace(_replace(_replace(PLAIN, "2 1 2 0.25 0.25 0.25", "2 1 3 0.25 0.25 0.25"),
                                  "4 2 2 0.25 0.75 0.25", "4 2 3 0.25 0.75 0.25"),
                         "2 atom types", "3 atom types"),
    "type_exceeds_declared": _replace(PLAIN, "2 atom types", "1 atom types"),
    "non_numeric": _replace(PLAIN, "0.75 0.75 0.75", "0.75 x 0.75"),
    "non_finite": _replace(PLAIN, "0.75 0.75 0.75", "0.75 nan 0.75"),
    "type_labels": PLAIN + "\nAtom Type Labels\n\n1 A\n2 B\n",
    "ellipsoids": PLAIN + "\nEllipsoids\n\n1 1 1 1 1 0 0 0\n",
    "impropers": _replace(CHAIN, "1 dihedral types\n", "1 dihedral types\n1 impropers\n"),
    "duplicate_section": CHAIN + "\nMasses\n\n1 1.0\n",
    "velocities_missing_atom": _replace(CHAIN, "6 0.0 0.0 -0.3\n", ""),
    "velocities_unknown_atom": _replace(CHAIN, "6 0.0 0.0 -0.3", "9 0.0 0.0 -0.3"),
    "masses_missing_type": _replace(CHAIN, "3 0.75\n", ""),
    "mass_not_positive": _replace(CHAIN, "3 0.75", "3 -0.75"),
    "bond_unknown_atom": _replace(CHAIN, "4 1 5 6\n", "4 1 5 9\n"),
    "bond_count_mismatch": _replace(CHAIN, "4 bonds", "5 bonds"),
    "bond_bad_width": _replace(CHAIN, "4 1 5 6\n", "4 1 5\n"),
    "bond_duplicate_id": _replace(CHAIN, "4 1 5 6\n", "3 1 5 6\n"),
    "title_ending_in_a_count_word": _replace(PLAIN, "four beads in a unit box",
                                             "plain atoms"),
    "angle_type_gap": _replace(CHAIN, "2 1 2 3 4\n", "2 3 2 3 4\n").replace(
        "1 angle types", "3 angle types"),
}


def _trajectory_bytes() -> bytes:
    """Two frames, five particles, every field, in a slot order that is not
    the tag order (float32 reals)."""
    n = 5
    rec = np.dtype([("tag", "<u4"), ("type", "<i4"), ("position", "<f4", (3,)),
                    ("image", "<i4", (3,)), ("velocity", "<f4", (3,)), ("force", "<f4", (3,))])
    units = b"reduced"
    head = b"BEADS_TRAJECTORY" + struct.pack("<II", 1, 0x01020304)
    head += struct.pack("<IIIII", 4, 4, 4, 4, 4)
    head += struct.pack("<Q", len(units)) + units
    head += struct.pack("<IQQ", 63, n, rec.itemsize)
    rng = np.random.default_rng(4)
    body = b""
    for step in (0, 50):
        recs = np.zeros(n, rec)
        recs["tag"] = [3, 1, 5, 2, 4]
        recs["type"] = [1, 2, 1, 1, 2]
        recs["position"] = rng.uniform(0.0, 10.0, (n, 3)).astype(np.float32)
        recs["image"] = rng.integers(-2, 3, (n, 3))
        recs["velocity"] = rng.normal(size=(n, 3)).astype(np.float32)
        recs["force"] = (rng.normal(size=(n, 3)) * 1e3).astype(np.float32)
        body += struct.pack("<Q", step) + np.array([[0, 0, 0], [10, 10, 10]],
                                                   "<f4").tobytes() + recs.tobytes()
    return head + body


def main(reference: str) -> None:
    sys.path.insert(0, str(pathlib.Path(reference) / "python"))
    from beads import io as ref_io  # the reference's own package

    OUT.mkdir(exist_ok=True)
    expect: dict = {"valid": {}, "invalid": {}, "dumps": {}}
    for name, text in (("chain", CHAIN), ("plain", PLAIN)):
        path = OUT / f"{name}.data"
        path.write_text(text)
        s = ref_io.read_lammps_data(path, units="reduced")
        arrays = {k: np.asarray(getattr(s, k)) for k in
                  ("positions", "box_bound", "types", "velocities", "masses", "tags",
                   "molecule_ids", "images")}
        np.savez(OUT / f"{name}.npz", **arrays)
        expect["valid"][name] = {"bonds": [list(b) for b in s.topology.bonds],
                                 "angles": [list(a) for a in s.topology.angles],
                                 "dihedrals": [list(d) for d in s.topology.dihedrals]}
    for name, text in INVALID.items():
        path = OUT / f"bad_{name}.data"
        path.write_text(text)
        try:
            ref_io.read_lammps_data(path, units="reduced")
        except Exception as exc:  # noqa: BLE001 - recording what the reference raises
            expect["invalid"][name] = [type(exc).__name__, str(exc)]
        else:
            raise SystemExit(f"the reference accepted {name}")
    traj = OUT / "traj.beadsbin"
    traj.write_bytes(_trajectory_bytes())
    for label, kwargs in (("sorted_17", {}), ("slot_order_6",
                                             {"sort_by_tag": False, "precision": 6})):
        ref_io.write_lammps_dump(traj, OUT / f"{label}.dump", **kwargs)
        expect["dumps"][label] = kwargs
    (OUT / "expect.json").write_text(json.dumps(expect, indent=1, sort_keys=True))
    print("wrote", sorted(p.name for p in OUT.iterdir()))


if __name__ == "__main__":
    main(sys.argv[1])
