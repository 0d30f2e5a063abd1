"""ctypes front end of the CPU oracle (``liboracle.so``).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine and the CPU arm of
the benchmark.  Nothing in ``beads_b200`` imports this module.

Every function takes NumPy arrays in particle-row order.  Bonded records are
given with 1-based tags as in the public API and are converted to rows here
(rows are tag - 1, so inputs must be tag-ordered).
"""

from __future__ import annotations

import ctypes
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")

_lib = None


def build() -> pathlib.Path:
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = ctypes.CDLL(str(LIB_PATH))
        _declare(_lib)
    return _lib


def _declare(L) -> None:
    c = ctypes
    L.orc_plan.argtypes = [_f32p, _f32p, c.c_double, c.c_double, _u32p, _f32p,
                           c.POINTER(c.c_float), c.POINTER(c.c_int)]
    L.orc_plan.restype = c.c_int
    L.orc_cell_ids.argtypes = [c.c_uint32, _f32p, _f32p, _f32p, c.c_double, c.c_double, _u32p]
    L.orc_cell_ids.restype = None
    L.orc_exclusions.argtypes = [c.c_uint32, c.c_void_p, c.c_uint32, c.c_uint32,
                                 c.c_void_p, c.c_uint64]
    L.orc_exclusions.restype = c.c_int64
    L.orc_neighbors.argtypes = [c.c_uint32, _f32p, _f32p, _f32p, c.c_double, c.c_double,
                                c.c_void_p, c.c_void_p, c.c_uint32, _u32p, _u32p]
    L.orc_neighbors.restype = c.c_int
    bonded = [c.c_uint32, c.c_void_p, c.c_void_p, c.c_void_p,
              c.c_uint32, c.c_void_p, c.c_void_p, c.c_void_p,
              c.c_uint32, c.c_void_p, c.c_void_p, c.c_void_p, c.c_void_p]
    L.orc_forces.argtypes = [c.c_uint32, _f32p, _i32p, _f32p, _f32p, c.c_int, _f64p, _f64p,
                             c.c_double, c.c_int, c.c_double, c.c_int, *bonded,
                             _f64p, _f64p, c.POINTER(c.c_double)]
    L.orc_forces.restype = c.c_int
    L.orc_sim_create.argtypes = [c.c_uint32, _f64p, _f64p, _f64p, c.c_void_p, _i32p, _f32p,
                                 _f32p, c.c_int, _f64p, _f64p, c.c_double, c.c_int,
                                 c.c_double, c.c_uint64, c.c_int, *bonded, c.c_double, c.c_int,
                                 c.c_double, c.c_double]
    L.orc_sim_create.restype = c.c_void_p
    L.orc_sim_destroy.argtypes = [c.c_void_p]
    L.orc_sim_destroy.restype = None
    L.orc_sim_step.argtypes = [c.c_void_p, c.c_uint64, _f64p]
    L.orc_sim_step.restype = None
    L.orc_sim_minimize.argtypes = [c.c_void_p, c.c_uint32, c.c_double, c.c_double]
    L.orc_sim_minimize.restype = None
    L.orc_sim_state.argtypes = [c.c_void_p, _f64p, _f64p, _i32p, c.POINTER(c.c_uint64)]
    L.orc_sim_state.restype = None
    L.orc_num_threads.argtypes = []
    L.orc_num_threads.restype = c.c_int


def _box(box_bound):
    bb = np.asarray(box_bound, dtype=np.float32).reshape(2, 3)
    return np.ascontiguousarray(bb[0]), np.ascontiguousarray(bb[1])


def _ptr(a):
    return None if a is None else a.ctypes.data


def plan(box_bound, cutoff: float, skin: float) -> dict:
    lo, hi = _box(box_bound)
    nc = np.zeros(3, np.uint32)
    inv = np.zeros(3, np.float32)
    sq = ctypes.c_float()
    path = ctypes.c_int()
    rc = lib().orc_plan(lo, hi, cutoff, skin, nc, inv, ctypes.byref(sq), ctypes.byref(path))
    if rc != 0:
        raise ValueError("neighbor search_cutoff must not exceed half shortest box length.")
    return {"nc": nc, "inv_cell": inv, "search_sq": sq.value,
            "path": ("direct", "regular_cell", "small_dimension")[path.value]}


def cell_ids(positions, box_bound, cutoff: float, skin: float) -> np.ndarray:
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    lo, hi = _box(box_bound)
    out = np.zeros(pos.shape[0], np.uint32)
    lib().orc_cell_ids(pos.shape[0], pos, lo, hi, cutoff, skin, out)
    return out


def exclusion_pairs(n: int, bonds, distance: int) -> np.ndarray:
    """Excluded pairs as 0-based rows (i < j), bonds given with 1-based tags."""
    rows = _bond_rows(bonds)
    nb = rows.shape[0]
    cnt = lib().orc_exclusions(n, _ptr(rows), nb, distance, None, 0)
    out = np.zeros((max(cnt, 0), 2), np.uint32)
    lib().orc_exclusions(n, _ptr(rows), nb, distance, _ptr(out), cnt)
    return out


def _exclusion_csr(n: int, bonds, distance: int):
    pairs = exclusion_pairs(n, bonds, distance)
    rows = [[] for _ in range(n)]
    for i, j in pairs.tolist():
        rows[i].append(j)
        rows[j].append(i)
    off = np.zeros(n + 1, np.uint32)
    off[1:] = np.cumsum([len(r) for r in rows])
    idx = np.array([j for r in rows for j in r], dtype=np.uint32)
    return off, idx


def neighbors(positions, box_bound, cutoff: float, skin: float, *, bonds=None,
              exclusion_distance: int = 0, cap: int = 1024):
    """Full neighbour sets (sorted rows) by the reference inclusion rule."""
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    n = pos.shape[0]
    lo, hi = _box(box_bound)
    off = idx = None
    if exclusion_distance and bonds is not None and len(bonds):
        off, idx = _exclusion_csr(n, bonds, exclusion_distance)
        if idx.size == 0:
            idx = np.zeros(1, np.uint32)
    counts = np.zeros(n, np.uint32)
    partners = np.zeros(n * cap, np.uint32)
    rc = lib().orc_neighbors(n, pos, lo, hi, cutoff, skin, _ptr(off), _ptr(idx), cap, counts,
                             partners)
    if rc != 0:
        raise ValueError("neighbor search_cutoff must not exceed half shortest box length.")
    partners = partners.reshape(n, cap)
    return counts, partners


def _bond_rows(bonds):
    if bonds is None or len(bonds) == 0:
        return np.zeros((0, 3), np.uint32)
    b = np.ascontiguousarray(bonds, dtype=np.uint32).reshape(-1, 3).copy()
    b[:, :2] -= 1
    return b


def _term_rows(records, width):
    if records is None or len(records) == 0:
        return np.zeros((0, width), np.uint32)
    r = np.ascontiguousarray(records, dtype=np.uint32).reshape(-1, width).copy()
    r[:, : width - 1] -= 1
    return r


def _coeff(arr, dtype):
    return None if arr is None else np.ascontiguousarray(arr, dtype=dtype)


class ForceField:
    """Plain container of the force-field tables the oracle needs."""

    def __init__(self, *, epsilon, sigma, cutoff, shift=False, bond_k=None, bond_r0=None,
                 angle_k=None, angle_theta0=None, dihedral_k=None, dihedral_d=None,
                 dihedral_n=None, exclusion_distance=0):
        self.epsilon = np.ascontiguousarray(epsilon, dtype=np.float64)
        self.sigma = np.ascontiguousarray(sigma, dtype=np.float64)
        self.ntypes = int(round(np.sqrt(self.epsilon.size)))
        self.cutoff = float(cutoff)
        self.shift = bool(shift)
        self.bond_k = _coeff(bond_k, np.float64)
        self.bond_r0 = _coeff(bond_r0, np.float64)
        self.angle_k = _coeff(angle_k, np.float64)
        self.angle_theta0 = _coeff(angle_theta0, np.float64)
        self.dihedral_k = _coeff(dihedral_k, np.float64)
        self.dihedral_d = _coeff(dihedral_d, np.int32)
        self.dihedral_n = _coeff(dihedral_n, np.int32)
        self.exclusion_distance = int(exclusion_distance)


def _bonded_args(ff: ForceField, bonds, angles, dihedrals):
    b = _bond_rows(bonds)
    a = _term_rows(angles, 4)
    d = _term_rows(dihedrals, 5)
    keep = [b, a, d]
    args = [b.shape[0], _ptr(b) if b.size else None, _ptr(ff.bond_k), _ptr(ff.bond_r0),
            a.shape[0], _ptr(a) if a.size else None, _ptr(ff.angle_k), _ptr(ff.angle_theta0),
            d.shape[0], _ptr(d) if d.size else None, _ptr(ff.dihedral_k), _ptr(ff.dihedral_d),
            _ptr(ff.dihedral_n)]
    return args, keep


def forces(positions, types, box_bound, ff: ForceField, *, skin: float = 0.0, bonds=None,
           angles=None, dihedrals=None):
    """FP64 forces [n,3], energies (pair, bond, angle, dihedral) and virial."""
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    ty = np.ascontiguousarray(types, dtype=np.int32)
    n = pos.shape[0]
    lo, hi = _box(box_bound)
    f = np.zeros(3 * n, np.float64)
    e = np.zeros(4, np.float64)
    w = ctypes.c_double()
    args, _keep = _bonded_args(ff, bonds, angles, dihedrals)
    rc = lib().orc_forces(n, pos, ty, lo, hi, ff.ntypes, ff.epsilon, ff.sigma, ff.cutoff,
                          int(ff.shift), skin, ff.exclusion_distance, *args, f, e,
                          ctypes.byref(w))
    if rc != 0:
        raise ValueError("neighbor search_cutoff must not exceed half shortest box length.")
    return f.reshape(n, 3), e, w.value


class Sim:
    """Persistent FP64 velocity-Verlet (+ Berendsen) state with the reference's
    step order and rebuild policy; ``step(k)`` advances k MD steps."""

    def __init__(self, positions, velocities, masses, types, box_bound, ff: ForceField, *,
                 dt: float, skin: float = 0.3, check_every: int = 1, images=None, bonds=None,
                 angles=None, dihedrals=None, thermostat: bool = False, kt_target: float = 0.0,
                 tau: float = 1.0):
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1)
        vel = np.ascontiguousarray(velocities, dtype=np.float64).reshape(-1)
        self.n = pos.size // 3
        mass = np.ascontiguousarray(masses, dtype=np.float64)
        img = (None if images is None
               else np.ascontiguousarray(images, dtype=np.int32).reshape(-1))
        ty = np.ascontiguousarray(types, dtype=np.int32)
        lo, hi = _box(box_bound)
        args, keep = _bonded_args(ff, bonds, angles, dihedrals)
        self._keep = keep
        self._h = lib().orc_sim_create(self.n, pos, vel, mass, _ptr(img), ty, lo, hi, ff.ntypes,
                                       ff.epsilon, ff.sigma, ff.cutoff, int(ff.shift), skin,
                                       check_every, ff.exclusion_distance, *args, dt,
                                       int(thermostat), kt_target, tau)
        if not self._h:
            raise ValueError("neighbor search_cutoff must not exceed half shortest box length.")

    def step(self, steps: int) -> np.ndarray:
        """Advance; returns [step, pair, bond, angle, dihedral, ke, virial]."""
        obs = np.zeros(7, np.float64)
        lib().orc_sim_step(self._h, int(steps), obs)
        return obs

    def minimize(self, iterations: int, dmax: float, fref: float) -> None:
        """Capped steepest descent of the positions (the engine's relaxation
        of random starts, in double); counters restart afterwards."""
        lib().orc_sim_minimize(self._h, int(iterations), float(dmax), float(fref))

    def state(self):
        pos = np.zeros(3 * self.n, np.float64)
        vel = np.zeros(3 * self.n, np.float64)
        img = np.zeros(3 * self.n, np.int32)
        builds = ctypes.c_uint64()
        lib().orc_sim_state(self._h, pos, vel, img, ctypes.byref(builds))
        return pos.reshape(-1, 3), vel.reshape(-1, 3), img.reshape(-1, 3), int(builds.value)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().orc_sim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def md(positions, velocities, masses, types, box_bound, ff: ForceField, *, dt: float,
       steps: int, skin: float = 0.3, check_every: int = 1, images=None, bonds=None,
       angles=None, dihedrals=None, thermostat: bool = False, kt_target: float = 0.0,
       tau: float = 1.0, obs_every: int = 0):
    """FP64 trajectory.  Returns (positions, velocities, images, thermo rows
    [step, pair, bond, angle, dihedral, ke, virial] every obs_every steps from
    step 0, build count)."""
    sim = Sim(positions, velocities, masses, types, box_bound, ff, dt=dt, skin=skin,
              check_every=check_every, images=images, bonds=bonds, angles=angles,
              dihedrals=dihedrals, thermostat=thermostat, kt_target=kt_target, tau=tau)
    rows = []
    if obs_every:
        rows.append(sim.step(0))
        done = 0
        while done < steps:
            k = min(obs_every, steps - done)
            obs = sim.step(k)
            done += k
            if done % obs_every == 0:
                rows.append(obs)
    else:
        sim.step(steps)
    pos, vel, img, builds = sim.state()
    sim.close()
    return pos, vel, img, np.array(rows).reshape(-1, 7), builds


def num_threads() -> int:
    return int(lib().orc_num_threads())
