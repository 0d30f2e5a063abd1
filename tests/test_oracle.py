"""The CPU oracle checked against independent arithmetic (CPU only).

* forces are minus the gradient of the oracle's own energy (central finite
  differences in double), for LJ and each harmonic term;
* neighbour sets equal an O(N^2) NumPy evaluation of the reference rule in
  float32;
* plan / cell ids follow the reference's float rules;
* bond-graph exclusions match hand-counted answers.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O


def _fd_check(pos, types, box, ff, bonds=None, angles=None, dihedrals=None, h=1e-4, tol=2e-3):
    """Central difference of total energy vs oracle force on a few atoms.

    Positions are float32 inside the oracle, so h is chosen large enough that
    the float rounding of pos +- h is negligible against the difference."""
    f, _, _ = O.forces(pos, types, box, ff, skin=0.3, bonds=bonds, angles=angles,
                       dihedrals=dihedrals)

    def energy(p):
        _, e, _ = O.forces(p, types, box, ff, skin=0.3, bonds=bonds, angles=angles,
                           dihedrals=dihedrals)
        return e.sum()

    rng = np.random.default_rng(0)
    for i in rng.choice(pos.shape[0], size=min(6, pos.shape[0]), replace=False):
        for a in range(3):
            p1 = pos.astype(np.float64).copy()
            p2 = p1.copy()
            p1[i, a] += h
            p2[i, a] -= h
            hp = np.float32(p1[i, a]) - np.float64(pos[i, a])
            hm = np.float64(pos[i, a]) - np.float32(p2[i, a])
            num = -(energy(p1.astype(np.float32)) - energy(p2.astype(np.float32))) / (hp + hm)
            assert abs(num - f[i, a]) <= tol * max(1.0, abs(f[i, a])), (i, a, num, f[i, a])


def _chain(n_beads=8, spacing=1.0, seed=0):
    rng = np.random.default_rng(seed)
    pos = np.zeros((n_beads, 3))
    pos[0] = [3.0, 3.0, 3.0]
    for k in range(1, n_beads):
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        pos[k] = pos[k - 1] + spacing * d
    return pos


def test_lj_forces_are_minus_energy_gradient():
    rng = np.random.default_rng(1)
    n = 64
    box = np.array([[0, 0, 0], [5.0, 5.0, 5.0]], np.float32)
    g = np.indices((4, 4, 4)).reshape(3, -1).T * 1.25 + 0.6
    pos = (g + rng.uniform(-0.1, 0.1, g.shape)).astype(np.float32)
    types = (np.arange(n) % 2 + 1).astype(np.int32)
    ff = O.ForceField(epsilon=[1.0, 0.7, 0.7, 0.5], sigma=[1.0, 0.94, 0.94, 0.88], cutoff=2.2,
                      shift=True)
    _fd_check(pos, types, box, ff)


@pytest.mark.parametrize("term", ["bond", "angle", "dihedral"])
def test_bonded_forces_are_minus_energy_gradient(term):
    pos = _chain(6, 1.0).astype(np.float32)
    box = np.array([[0, 0, 0], [12.0, 12.0, 12.0]], np.float32)
    types = np.ones(6, np.int32)
    bonds = [(k, k + 1, 1) for k in range(1, 6)]
    ff = O.ForceField(epsilon=[1e-9], sigma=[0.1], cutoff=0.2, bond_k=[50.0], bond_r0=[0.8],
                      angle_k=[5.0], angle_theta0=[110.0], dihedral_k=[1.5], dihedral_d=[-1],
                      dihedral_n=[3])
    kw = {"bonds": bonds}
    if term == "angle":
        kw["angles"] = [(k, k + 1, k + 2, 1) for k in range(1, 5)]
    if term == "dihedral":
        kw["dihedrals"] = [(k, k + 1, k + 2, k + 3, 1) for k in range(1, 4)]
    _fd_check(pos, types, box, ff, **kw)


def test_bonded_across_periodic_boundary_uses_minimum_image():
    box = np.array([[0, 0, 0], [6.0, 6.0, 6.0]], np.float32)
    pos = np.array([[5.9, 3.0, 3.0], [0.4, 3.1, 3.0]], np.float32)  # 0.5 apart through x
    ff = O.ForceField(epsilon=[1e-9], sigma=[0.1], cutoff=0.2, bond_k=[10.0], bond_r0=[1.0])
    f, e, w = O.forces(pos, np.ones(2, np.int32), box, ff, bonds=[(1, 2, 1)])
    r = np.hypot(0.5, 0.1)
    assert e[1] == pytest.approx(0.5 * 10.0 * (r - 1.0) ** 2, rel=1e-6)
    assert f[0, 0] < 0 and f[1, 0] > 0  # stretched bond pulls the pair together


def _brute_neighbors(pos, box, cutoff, skin, excluded=frozenset()):
    pos = np.asarray(pos, np.float32)
    lo = box[0].astype(np.float32)
    length = (box[1] - box[0]).astype(np.float32)
    half = np.float32(0.5) * length
    sc = np.float32(cutoff) + np.float32(skin)
    sc2 = sc * sc
    out = []
    for i in range(pos.shape[0]):
        d = (pos[i] - pos).astype(np.float32)
        d = np.where(d > half, d - length, np.where(d < -half, d + length, d)).astype(np.float32)
        # r^2 = fma(dz,dz, fma(dx,dx, dy*dy)): emulate the two fused steps exactly in float64.
        dy2 = (d[:, 1] * d[:, 1]).astype(np.float32)
        s1 = (d[:, 0].astype(np.float64) ** 2 + dy2.astype(np.float64)).astype(np.float32)
        r2 = (d[:, 2].astype(np.float64) ** 2 + s1.astype(np.float64)).astype(np.float32)
        js = [j for j in np.nonzero(r2 <= sc2)[0] if j != i and (min(i, j), max(i, j)) not in excluded]
        out.append(tuple(sorted(js)))
    return out


@pytest.mark.parametrize("lens", [(9.5, 9.5, 9.5), (6.1, 9.3, 6.1), (5.9, 5.9, 5.9)])
def test_neighbor_sets_match_bruteforce(lens):
    rng = np.random.default_rng(2)
    box = np.array([[0, 0, 0], lens], np.float32)
    n = int(0.8 * np.prod(lens))
    pos = (rng.uniform(0, 1, (n, 3)) * np.array(lens)).astype(np.float32)
    counts, partners = O.neighbors(pos, box, 2.5, 0.3, cap=256)
    ours = [tuple(partners[i, : counts[i]].tolist()) for i in range(n)]
    assert ours == _brute_neighbors(pos, box, 2.5, 0.3)


def test_neighbor_sets_skip_excluded_pairs():
    pos = _chain(10, 0.97, seed=3)
    pos = (pos - pos.min(axis=0) + 1.0).astype(np.float32)
    box = np.array([[0, 0, 0], [14.0, 14.0, 14.0]], np.float32)
    bonds = [(k, k + 1, 1) for k in range(1, 10)]
    counts, partners = O.neighbors(pos, box, 1.5, 0.3, bonds=bonds, exclusion_distance=2, cap=32)
    excl = {tuple(p) for p in O.exclusion_pairs(10, bonds, 2).tolist()}
    ours = [tuple(partners[i, : counts[i]].tolist()) for i in range(10)]
    assert ours == _brute_neighbors(pos, box, 1.5, 0.3, frozenset(excl))


def test_exclusion_pairs_known_answers():
    chain = [(k, k + 1, 1) for k in range(1, 6)]  # 6 beads
    assert O.exclusion_pairs(6, chain, 1).tolist() == [[0, 1], [1, 2], [2, 3], [3, 4], [4, 5]]
    assert len(O.exclusion_pairs(6, chain, 2)) == 5 + 4
    assert len(O.exclusion_pairs(6, chain, 3)) == 5 + 4 + 3
    # Ring of 4: distance 2 already covers every pair once.
    ring = [(1, 2, 1), (2, 3, 1), (3, 4, 1), (4, 1, 1)]
    assert O.exclusion_pairs(4, ring, 2).tolist() == [[0, 1], [0, 2], [0, 3], [1, 2], [1, 3],
                                                      [2, 3]]
    # Star: the hub's leaves are two bonds apart from each other.
    star = [(1, k, 1) for k in range(2, 6)]
    assert len(O.exclusion_pairs(5, star, 1)) == 4
    assert len(O.exclusion_pairs(5, star, 2)) == 4 + 6


def test_plan_rules():
    p = O.plan([[0, 0, 0], [16.929, 16.929, 16.929]], 2.5, 0.3)
    assert p["nc"].tolist() == [6, 6, 6] and p["path"] == "regular_cell"
    p = O.plan([[0, 0, 0], [37.2, 37.2, 37.2]], 0.9, 0.1)
    assert p["nc"].tolist() == [37, 37, 37]
    p = O.plan([[0, 0, 0], [6.0, 6.0, 6.0]], 2.5, 0.3)
    assert p["nc"].tolist() == [2, 2, 2] and p["path"] == "direct"
    p = O.plan([[0, 0, 0], [9.0, 6.0, 9.0]], 2.5, 0.3)
    assert p["path"] == "small_dimension"
    with pytest.raises(ValueError):
        O.plan([[0, 0, 0], [5.0, 5.0, 5.0]], 2.5, 0.3)


def test_cell_ids_clamp_and_flatten():
    box = np.array([[0, 0, 0], [9.0, 9.0, 9.0]], np.float32)
    pos = np.array([[0.0, 0.0, 0.0], [8.999999, 0.0, 0.0], [0.0, 3.0, 0.0], [0.0, 0.0, 6.1]],
                   np.float32)
    cells = O.cell_ids(pos, box, 2.5, 0.3)
    assert cells.tolist() == [0, 2, 3, 18]


def test_md_conserves_energy_in_fp64():
    n_side = 6
    a = (1 / 0.8442) ** (1 / 3)
    g = np.indices((n_side,) * 3).reshape(3, -1).T * a + 0.5 * a
    rng = np.random.default_rng(4)
    pos = (g + rng.uniform(-0.05, 0.05, g.shape)).astype(np.float32)
    n = pos.shape[0]
    vel = rng.standard_normal((n, 3)) * 0.8
    vel -= vel.mean(axis=0)
    box = np.array([[0, 0, 0], [n_side * a] * 3], np.float32)
    # shift=True keeps the energy continuous at the cutoff (pairs crossing rc
    # would otherwise add jumps of U(rc) that are not integration error).
    ff = O.ForceField(epsilon=[1.0], sigma=[1.0], cutoff=2.5, shift=True)
    _, _, _, thermo, builds = O.md(pos, vel, np.ones(n), np.ones(n, np.int32), box, ff,
                                   dt=0.002, steps=400, skin=0.3, obs_every=50)
    etot = thermo[:, 1] + thermo[:, 5]
    assert np.ptp(etot) / n < 5e-3
    assert builds >= 2
