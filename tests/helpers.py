"""Glue between ReplicaSpec inputs and the CPU oracle used as the checker."""

from __future__ import annotations

import numpy as np

from oracle import oracle as O


def oracle_ff(spec) -> O.ForceField:
    return O.ForceField(
        epsilon=np.asarray(spec.epsilon, np.float64).ravel(),
        sigma=np.asarray(spec.sigma, np.float64).ravel(),
        cutoff=spec.cutoff, shift=spec.shift,
        bond_k=spec.bond_k, bond_r0=spec.bond_r0,
        angle_k=spec.angle_k, angle_theta0=spec.angle_theta0,
        dihedral_k=spec.dihedral_k, dihedral_d=spec.dihedral_d, dihedral_n=spec.dihedral_n,
        exclusion_distance=spec.exclusion_distance)


def oracle_forces(spec, positions=None):
    pos = spec.positions if positions is None else positions
    return O.forces(pos, spec.types, spec.box_bound, oracle_ff(spec),
                    skin=spec.cutoff_buffer, bonds=spec.bonds, angles=spec.angles,
                    dihedrals=spec.dihedrals)


def oracle_neighbors(spec, positions=None, cap=None):
    pos = spec.positions if positions is None else positions
    return O.neighbors(pos, spec.box_bound, spec.cutoff, spec.cutoff_buffer, bonds=spec.bonds,
                       exclusion_distance=spec.exclusion_distance,
                       cap=cap or int(spec.max_neighbors))


def rel_rms(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def neighbor_sets(counts, partners):
    """Sorted partner tuple per row (partners given as 1-based tags)."""
    return [tuple(sorted(int(x) for x in partners[i, : counts[i]])) for i in range(len(counts))]


def kinetic(vel, masses) -> float:
    v = np.asarray(vel, np.float64)
    return float(0.5 * (np.asarray(masses, np.float64)[:, None] * v * v).sum())


def mix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser of unsigned 64-bit values (wrapping arithmetic)."""
    z = np.asarray(x, np.uint64) + np.uint64(0x9E3779B97F4A7C15)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def partner_hash(counts, partners) -> np.ndarray:
    """Order-free hash of each row's partner set: sum of mix64(tag) over the
    first counts[i] entries of row i (tags 1-based), modulo 2^64."""
    counts = np.asarray(counts)
    partners = np.asarray(partners)
    cap = partners.shape[1]
    out = np.zeros(counts.shape[0], np.uint64)
    step = max(1, (1 << 24) // max(cap, 1))
    for a in range(0, counts.shape[0], step):
        b = min(counts.shape[0], a + step)
        z = mix64(partners[a:b].astype(np.uint64))
        z[np.arange(cap)[None, :] >= counts[a:b, None]] = 0
        with np.errstate(over="ignore"):
            out[a:b] = z.sum(axis=1, dtype=np.uint64)
    return out


def partner_hash_all(hashes: np.ndarray) -> int:
    """One 64-bit value over every row's hash, tied to the row index."""
    rows = np.arange(1, np.asarray(hashes).shape[0] + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        return int(mix64(np.asarray(hashes, np.uint64) ^ mix64(rows)).sum(dtype=np.uint64))
