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
