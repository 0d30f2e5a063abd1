"""Seeded synthetic inputs with the shapes of the benchmark configurations.

No dataset is involved anywhere: every configuration is generated here from
fixed seeds.

* ``lj_lattice``      4,096-bead single-type LJ fluid on a jittered simple-cubic
                      lattice, reduced units (rho 0.8442, rc 2.5, skin 0.3).
* ``lj_mixture``      binary LJ mixture in nm_kjmol units (80/20 types, mass
                      39.95 u, rho 20.37 nm^-3), uniform random start that the
                      caller relaxes with ``Engine.minimize``.
* ``polymer_melt``    bead-spring chains (seeded random walks, step 0.97,
                      rejection radius 0.8) with harmonic bonds, angles and
                      dihedrals, reduced units, rho 0.85.
* ``replica_batch``   many independent single-type LJ boxes of uneven size.
* ``relaxed``         a spec moved by capped steepest descent on the GPU.

Each function returns ``ReplicaSpec`` objects for ``beads_b200.engine.Engine``.
"""

from __future__ import annotations

import math

import numpy as np

from .engine import ReplicaSpec

KB_NM_KJMOL = 0.00831446261815324


def _gaussian_velocities(rng, n, masses, kt):
    v = rng.standard_normal((n, 3)) * np.sqrt(kt / masses)[:, None]
    p = (v * masses[:, None]).sum(axis=0) / masses.sum()
    return (v - p).astype(np.float32)


def _inside(pos, lo, hi):
    """Wrap into [lo, hi) in float32 (guards the rounding edge x == hi)."""
    length = hi - lo
    pos = lo + np.mod(pos - lo, length)
    pos = pos.astype(np.float32)
    for a in range(3):
        over = pos[:, a] >= np.float32(hi[a])
        pos[over, a] = np.nextafter(np.float32(hi[a]), np.float32(lo[a]))
        under = pos[:, a] < np.float32(lo[a])
        pos[under, a] = np.float32(lo[a])
    return pos


def lj_lattice(n_side: int = 16, density: float = 0.8442, jitter: float = 0.05,
               temperature: float = 1.0, seed_pos: int = 1, seed_vel: int = 2,
               cutoff: float = 2.5, skin: float = 0.3, check_every: int = 10,
               dt: float = 0.005, max_neighbors: int = 512,
               sort_every_rebuild: int = 10) -> ReplicaSpec:
    a = (1.0 / density) ** (1.0 / 3.0)
    length = n_side * a
    g = np.indices((n_side,) * 3).reshape(3, -1).T.astype(np.float64)
    rng = np.random.default_rng(seed_pos)
    pos = (g + 0.5) * a + rng.uniform(-jitter, jitter, size=g.shape)
    lo = np.zeros(3)
    hi = np.full(3, length)
    pos = _inside(pos, lo, hi)
    n = pos.shape[0]
    masses = np.ones(n, np.float64)
    vel = _gaussian_velocities(np.random.default_rng(seed_vel), n, masses, temperature)
    return ReplicaSpec(
        positions=pos, types=np.ones(n, np.int32),
        box_bound=np.array([lo, hi], np.float32), epsilon=np.array([[1.0]]),
        sigma=np.array([[1.0]]), cutoff=cutoff, dt=dt, units="reduced", velocities=vel,
        masses=masses.astype(np.float32), shift=False, cutoff_buffer=skin,
        rebuild_check_every=check_every, max_neighbors=max_neighbors,
        sort_every_rebuild=sort_every_rebuild)


MIXTURE_EPS = np.array([[1.0, 0.7], [0.7, 0.5]])
MIXTURE_SIG = np.array([[0.34, 0.32], [0.32, 0.30]])


def lj_mixture(n: int = 1_048_576, box: float | None = 37.2, density: float | None = None,
               seed: int = 3, temperature: float = 120.0, tau: float = 0.1, dt: float = 0.002,
               skin: float = 0.1, max_neighbors: int = 128, sort_every_rebuild: int = 1,
               check_every: int = 1) -> ReplicaSpec:
    """Binary mixture (nm_kjmol).  ``box`` wins over ``density`` when given."""
    if box is None:
        box = (n / density) ** (1.0 / 3.0)
    rng = np.random.default_rng(seed)
    lo = np.zeros(3)
    hi = np.full(3, box)
    pos = _inside(rng.uniform(0.0, box, size=(n, 3)), lo, hi)
    types = np.ones(n, np.int32)
    types[rng.permutation(n)[: int(round(0.2 * n))]] = 2
    masses = np.full(n, 39.95)
    vel = _gaussian_velocities(np.random.default_rng(seed + 1), n, masses,
                               KB_NM_KJMOL * temperature)
    return ReplicaSpec(
        positions=pos, types=types, box_bound=np.array([lo, hi], np.float32),
        epsilon=MIXTURE_EPS, sigma=MIXTURE_SIG, cutoff=0.9, dt=dt, units="nm_kjmol",
        velocities=vel, masses=masses.astype(np.float32), shift=True, cutoff_buffer=skin,
        rebuild_check_every=check_every, max_neighbors=max_neighbors,
        sort_every_rebuild=sort_every_rebuild, thermostat=(temperature, tau))


def _sequential_walks(rng, n_chains: int, beads: int, length: float, step: float,
                      reject: float) -> np.ndarray:
    """Chains grown one after another, bead by bead (pure Python; small melts)."""
    n = n_chains * beads
    cell = reject
    ncell = max(1, int(length // cell))
    grid: dict[tuple[int, int, int], list[int]] = {}
    pos = np.zeros((n, 3))

    def key(p):
        return tuple(int(c) % ncell for c in np.floor(p / (length / ncell)))

    def clash(p):
        kx, ky, kz = key(p)
        near = [j for dx in (-1, 0, 1) for dy in (-1, 0, 1) for dz in (-1, 0, 1)
                for j in grid.get(((kx + dx) % ncell, (ky + dy) % ncell, (kz + dz) % ncell), ())]
        if not near:
            return False
        d = p - pos[near]
        d -= length * np.round(d / length)
        return bool(((d * d).sum(axis=1) < reject * reject).any())

    def place(p, at):
        pos[at] = p
        grid.setdefault(key(p), []).append(at)

    def unplace(at):
        grid[key(pos[at])].remove(at)

    # Every bead keeps at least `reject` from every bead placed before it.  A
    # walk that finds no free direction in 200 tries backs off a few beads;
    # after 50 back-offs the chain restarts from a new random point.
    idx = 0
    for _ in range(n_chains):
        start, backoffs = idx, 0
        while idx < start + beads:
            if idx == start:
                while True:
                    p = rng.uniform(0.0, length, 3)
                    if not clash(p):
                        break
                place(p, idx)
                idx += 1
                continue
            for _attempt in range(200):
                u = rng.standard_normal(3)
                u /= np.linalg.norm(u)
                cand = np.mod(pos[idx - 1] + step * u, length)
                if not clash(cand):
                    place(cand, idx)
                    idx += 1
                    break
            else:
                backoffs += 1
                back = idx - start if backoffs > 50 else min(idx - start - 1, 4)
                if backoffs > 50:
                    backoffs = 0
                for _k in range(back):
                    idx -= 1
                    unplace(idx)
    return pos


# Offsets of a cell's 27-cell neighbourhood.
_STENCIL = np.array([(dx, dy, dz) for dx in (-1, 0, 1) for dy in (-1, 0, 1)
                     for dz in (-1, 0, 1)], np.int64)


def _lockstep_walks(rng, n_chains: int, beads: int, length: float, step: float,
                    reject: float) -> np.ndarray:
    """All chains grown together, at most one bead per chain per round (vectorised).

    Same acceptance rule as the sequential walk: a bead keeps at least
    ``reject`` from every bead already placed.  In a round, each unfinished
    chain proposes one bead (a uniform point for a chain's first bead, else a
    step of length ``step`` in a uniform direction from its last bead); a
    proposal is kept when it clears the placed beads and every proposal of a
    lower-numbered chain in the same round.  A chain makes several proposals a
    round (more as fewer chains remain) and keeps its first clear one.  A chain
    refused 200 times in a row backs off up to 4 beads, and after 50 back-offs
    it starts again.
    """
    from scipy.spatial import cKDTree

    n = n_chains * beads
    ncell = max(1, int(length // reject))
    csize = length / ncell
    # Points at least `reject` apart in a cube of side below 2 * reject / sqrt(3)
    # number at most 8 (one per octant); coarser grids (tiny boxes) get room for 64.
    cap = 8 if csize < 2.0 * reject / math.sqrt(3.0) else 64
    members = np.full((ncell ** 3, cap), -1, np.int32)
    fill = np.zeros(ncell ** 3, np.int64)
    # flat ids of every cell's 27-cell neighbourhood, periodic
    axis = np.arange(ncell)
    kk = np.stack(np.meshgrid(axis, axis, axis, indexing="ij"), -1).reshape(-1, 3)[:, ::-1]
    around = (kk[:, None, :] + _STENCIL[None, :, :]) % ncell
    stencil_of = ((around[..., 2] * ncell + around[..., 1]) * ncell
                  + around[..., 0]).astype(np.int32)
    del kk, around
    cell_of = np.full(n, -1, np.int64)
    pos = np.zeros((n, 3))
    size = np.zeros(n_chains, np.int64)
    refused = np.zeros(n_chains, np.int64)
    backoffs = np.zeros(n_chains, np.int64)
    r2 = reject * reject

    def cell_index(p):
        k = np.floor(p / csize).astype(np.int64) % ncell
        return (k[:, 2] * ncell + k[:, 1]) * ncell + k[:, 0]

    def unplace(at: int) -> None:
        c = cell_of[at]
        row = members[c]
        j = int(np.nonzero(row == at)[0][0])
        last = fill[c] - 1
        row[j] = row[last]
        row[last] = -1
        fill[c] = last
        cell_of[at] = -1

    while True:
        active = np.nonzero(size < beads)[0]
        if active.size == 0:
            break
        m = active.size
        tries = int(min(64, max(2, 8192 // m)))  # proposals per chain this round
        first = size[active] == 0
        cand = np.empty((m, tries, 3))
        cand[first] = rng.uniform(0.0, length, (int(first.sum()), tries, 3))
        grow = ~first
        if grow.any():
            u = rng.standard_normal((int(grow.sum()), tries, 3))
            u /= np.linalg.norm(u, axis=2)[..., None]
            prev = active[grow] * beads + size[active[grow]] - 1
            cand[grow] = pos[prev][:, None, :] + step * u
        cand = np.mod(cand, length).reshape(m * tries, 3)
        cand[cand >= length] = 0.0
        flat = cell_index(cand)
        who = members[stencil_of[flat]].reshape(m * tries, -1)
        row, col = np.nonzero(who >= 0)
        d = cand[row] - pos[who[row, col]]
        d -= length * np.round(d / length)
        hit = row[np.einsum("ij,ij->i", d, d) < r2]
        free = np.ones(m * tries, bool)
        free[hit] = False
        free = free.reshape(m, tries)
        # Each chain takes its first free proposal; `used` counts the attempts.
        pick = np.argmax(free, axis=1)
        found = free[np.arange(m), pick]
        used = np.where(found, pick + 1, tries)
        choice = np.arange(m) * tries + pick
        clash = ~found
        ok = np.nonzero(found)[0]
        if ok.size > 1:
            pts = cand[choice[ok]]
            pairs = cKDTree(pts, boxsize=length).query_pairs(reject, output_type="ndarray")
            if len(pairs):
                # Every proposal in a close pair but the lowest-numbered chain's
                # one is refused (proposals are in chain order).
                keep = np.ones(ok.size, bool)
                order = np.argsort(pairs[:, 0], kind="stable")
                for a, b in pairs[order]:
                    if keep[a]:
                        keep[b] = False
                clash[ok[~keep]] = True
                ok = ok[keep]
        if ok.size:
            chains = active[ok]
            at = chains * beads + size[chains]
            pos[at] = cand[choice[ok]]
            cells = flat[choice[ok]]
            srt = np.argsort(cells, kind="stable")
            cells_s = cells[srt]
            starts = np.r_[0, np.nonzero(np.diff(cells_s))[0] + 1]
            rank = np.arange(cells_s.size) - np.repeat(starts, np.diff(np.r_[starts,
                                                                            cells_s.size]))
            slot = fill[cells_s] + rank
            if slot.max() >= cap:
                raise RuntimeError("polymer_melt: cell capacity exceeded")
            members[cells_s, slot] = at[srt]
            np.add.at(fill, cells_s, 1)
            cell_of[at] = cells
            size[chains] += 1
            refused[chains] = 0
        bad = active[clash]
        refused[bad] += used[clash]
        for c in bad[refused[bad] >= 200]:
            refused[c] = 0
            backoffs[c] += 1
            if backoffs[c] > 50:
                back, backoffs[c] = int(size[c]), 0
            else:
                back = int(min(size[c] - 1, 4))
            for _k in range(back):
                size[c] -= 1
                unplace(int(c * beads + size[c]))
    return pos


def polymer_melt(n_chains: int = 2000, beads: int = 200, density: float = 0.85, seed: int = 5,
                 step: float = 0.97, reject: float = 0.8, temperature: float = 1.0,
                 tau: float = 1.0, dt: float = 0.005, skin: float = 0.3,
                 exclusion_distance: int = 2, dihedrals: bool = True,
                 max_neighbors: int = 128, growth: str = "sequential") -> ReplicaSpec:
    """Bead-spring melt from seeded self-avoiding random walks.

    ``growth="sequential"`` grows the chains one after another (the layout
    the small test melts are pinned on); ``"lockstep"`` grows them all
    together, vectorised, for melts of hundreds of thousands of beads.
    """
    n = n_chains * beads
    length = (n / density) ** (1.0 / 3.0)
    rng = np.random.default_rng(seed)
    if growth == "sequential":
        pos = _sequential_walks(rng, n_chains, beads, length, step, reject)
    elif growth == "lockstep":
        pos = _lockstep_walks(rng, n_chains, beads, length, step, reject)
    else:
        raise ValueError(f"unknown growth {growth!r}")
    lo = np.zeros(3)
    hi = np.full(3, length)
    posf = _inside(pos, lo, hi)
    tags = np.arange(1, n + 1, dtype=np.uint32)
    bonds, angles, dihs = [], [], []
    for c in range(n_chains):
        first = c * beads + 1
        for b in range(beads - 1):
            bonds.append((first + b, first + b + 1, 1))
        for b in range(beads - 2):
            angles.append((first + b, first + b + 1, first + b + 2, 1))
        if dihedrals:
            for b in range(beads - 3):
                dihs.append((first + b, first + b + 1, first + b + 2, first + b + 3, 1))
    masses = np.ones(n)
    vel = _gaussian_velocities(np.random.default_rng(seed + 1), n, masses, temperature)
    mol = np.repeat(np.arange(1, n_chains + 1, dtype=np.uint32), beads)
    return ReplicaSpec(
        positions=posf, types=np.ones(n, np.int32), box_bound=np.array([lo, hi], np.float32),
        epsilon=np.array([[1.0]]), sigma=np.array([[1.0]]), cutoff=2.0 ** (1.0 / 6.0), dt=dt,
        units="reduced", velocities=vel, masses=masses.astype(np.float32), tags=tags,
        molecule_ids=mol, shift=True, bonds=np.array(bonds, np.uint32),
        angles=np.array(angles, np.uint32),
        dihedrals=np.array(dihs, np.uint32) if dihedrals else None,
        bond_k=[500.0], bond_r0=[0.97], angle_k=[5.0], angle_theta0=[150.0],
        dihedral_k=[1.0] if dihedrals else None, dihedral_d=[1] if dihedrals else None,
        dihedral_n=[1] if dihedrals else None, exclusion_distance=exclusion_distance,
        cutoff_buffer=skin, max_neighbors=max_neighbors, thermostat=(temperature, tau))


def relaxed(spec: ReplicaSpec, iterations: int = 500, dmax: float = 0.01,
            fref: float = 100.0, capacity: int = 256) -> ReplicaSpec:
    """A copy of ``spec`` moved by ``iterations`` capped steepest-descent
    steps on the GPU (``Engine.minimize``: every bead moves dmax * F /
    max(|F|, fref), all force terms included), with positions wrapped into
    the box and images carried.  The descent runs with a list capacity of at
    least ``capacity``; the copy keeps the spec's own.  A start grown with a
    rejection radius below the pair minimum (the polymer melt: 0.8 against
    2^(1/6)) needs it before MD: from the raw start the overlapping pairs
    heat the melt until its neighbour lists overflow."""
    import dataclasses

    from .engine import Engine

    work = dataclasses.replace(spec, max_neighbors=max(capacity, spec.max_neighbors))
    with Engine(work) as eng:
        eng.minimize(iterations, dmax, fref)
        st = eng.state()
    box = np.asarray(spec.box_bound, np.float64)
    return dataclasses.replace(spec, positions=_inside(st["positions"].astype(np.float64),
                                                       box[0], box[1]),
                               images=st["images"].copy())


def replica_batch(n_replicas: int = 512, n_min: int = 256, n_max: int = 32768, seed: int = 7,
                  cutoff: float = 2.5, skin: float = 0.3, dt: float = 0.005,
                  max_neighbors: int = 160) -> list[ReplicaSpec]:
    """Uneven single-type LJ replicas: log-uniform sizes, rho ~ U[0.7, 0.9],
    Berendsen target T ~ U[0.8, 1.5] (tau 1), jittered lattices."""
    rng = np.random.default_rng(seed)
    out = []
    for r in range(n_replicas):
        n_target = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        rho = rng.uniform(0.7, 0.9)
        t_target = rng.uniform(0.8, 1.5)
        n = n_target
        side = int(math.ceil(n ** (1.0 / 3.0)))
        length = (n / rho) ** (1.0 / 3.0)
        length = max(length, 2.0 * (cutoff + skin) + 1e-3)
        a = length / side
        rr = np.random.default_rng(seed * 100003 + r)
        g = np.indices((side,) * 3).reshape(3, -1).T.astype(np.float64)
        g = g[np.sort(rr.permutation(g.shape[0])[:n])]
        pos = _inside((g + 0.5) * a + rr.uniform(-0.05, 0.05, g.shape), np.zeros(3),
                      np.full(3, length))
        masses = np.ones(n)
        vel = _gaussian_velocities(rr, n, masses, t_target)
        out.append(ReplicaSpec(
            positions=pos, types=np.ones(n, np.int32),
            box_bound=np.array([np.zeros(3), np.full(3, length)], np.float32),
            epsilon=np.array([[1.0]]), sigma=np.array([[1.0]]), cutoff=cutoff, dt=dt,
            units="reduced", velocities=vel, masses=masses.astype(np.float32),
            cutoff_buffer=skin, max_neighbors=max_neighbors, thermostat=(t_target, 1.0)))
    return out


def fit_mixture(n_replicas: int = 64, n: int = 8192, density: float = 0.8,
                temperature: float = 1.0, tau: float = 1.0, dt: float = 0.005, seed: int = 21,
                skin: float = 0.3, max_neighbors: int = 192) -> list[ReplicaSpec]:
    """Replicas of the binary mixture in reduced units (sigma11 = 1: the
    nm_kjmol mixture's tables divided by 0.34 nm, eps in kJ/mol as reduced
    energies), 80/20 types, jittered simple-cubic lattice start, Berendsen."""
    sig = MIXTURE_SIG / 0.34
    out = []
    side = int(math.ceil(n ** (1.0 / 3.0)))
    length = (n / density) ** (1.0 / 3.0)
    for r in range(n_replicas):
        rng = np.random.default_rng(seed * 1009 + r)
        g = np.indices((side,) * 3).reshape(3, -1).T.astype(np.float64)
        g = g[np.sort(rng.permutation(g.shape[0])[:n])]
        a = length / side
        pos = _inside((g + 0.5) * a + rng.uniform(-0.05, 0.05, g.shape), np.zeros(3),
                      np.full(3, length))
        types = np.ones(n, np.int32)
        types[rng.permutation(n)[: int(round(0.2 * n))]] = 2
        masses = np.ones(n)
        vel = _gaussian_velocities(rng, n, masses, temperature)
        out.append(ReplicaSpec(
            positions=pos, types=types,
            box_bound=np.array([np.zeros(3), np.full(3, length)], np.float32),
            epsilon=MIXTURE_EPS.copy(), sigma=sig, cutoff=0.9 / 0.34, dt=dt, units="reduced",
            velocities=vel, masses=masses.astype(np.float32), shift=True, cutoff_buffer=skin,
            max_neighbors=max_neighbors, sort_every_rebuild=10,
            thermostat=(temperature, tau)))
    return out

