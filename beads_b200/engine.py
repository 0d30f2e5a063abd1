"""Engine contexts over the C ABI: one or many replicas in one device batch.

``Engine`` is the in-process handle used by the benchmark, the tests and the
autograd wrapper; the public drop-in surface (``System`` / ``Simulation``)
goes through ``beads_b200._native.execute_simulation`` instead.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from . import _lib


@dataclass
class ReplicaSpec:
    """Everything one replica needs, as plain arrays and numbers.

    Bonded records use 1-based tags; ``epsilon``/``sigma`` are full symmetric
    ``n_types x n_types`` tables; ``thermostat`` is ``None`` or a
    ``(temperature, tau)`` pair in public units.
    """

    positions: np.ndarray
    types: np.ndarray
    box_bound: np.ndarray
    epsilon: np.ndarray
    sigma: np.ndarray
    cutoff: float
    dt: float
    units: str = "reduced"
    velocities: np.ndarray | None = None
    masses: np.ndarray | None = None
    tags: np.ndarray | None = None
    molecule_ids: np.ndarray | None = None
    images: np.ndarray | None = None
    shift: bool = False
    bonds: np.ndarray | None = None
    angles: np.ndarray | None = None
    dihedrals: np.ndarray | None = None
    bond_k: Sequence[float] | None = None
    bond_r0: Sequence[float] | None = None
    angle_k: Sequence[float] | None = None
    angle_theta0: Sequence[float] | None = None
    dihedral_k: Sequence[float] | None = None
    dihedral_d: Sequence[int] | None = None
    dihedral_n: Sequence[int] | None = None
    exclusion_distance: int = 0
    cutoff_buffer: float = 0.3
    rebuild_check_every: int = 1
    sort_every_rebuild: int = 10
    max_neighbors: int = 512
    thermostat: tuple[float, float] | None = None
    extra: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(np.asarray(self.positions).shape[0])

    @classmethod
    def from_spec(cls, spec: dict) -> "ReplicaSpec":
        """The replica a ``Simulation._native_spec()`` dict describes."""
        s, f, d, nb = spec["system"], spec["forcefield"], spec["dynamics"], spec["neighbor"]
        nt = int(np.asarray(s["types"]).max())
        eps = np.zeros((nt, nt))
        sig = np.zeros((nt, nt))
        for c in f["pair_coeffs"]:
            a, b = c["type_i"] - 1, c["type_j"] - 1
            eps[a, b] = eps[b, a] = c["params"]["epsilon"]
            sig[a, b] = sig[b, a] = c["params"]["sigma"]
        t = s["topology"]

        def recs(items, keys):
            return None if not items else np.array([[x[k] for k in keys] for x in items],
                                                   np.uint32)

        def coeffs(kind, key):
            cs = f.get(f"{kind}_coeffs") or []
            return [c["params"][key] for c in sorted(cs, key=lambda c: c["type"])] or None

        thermo = d.get("thermostat")
        return cls(
            positions=np.asarray(s["positions"]), types=np.asarray(s["types"]),
            box_bound=np.asarray(s["box_bound"]), epsilon=eps, sigma=sig,
            cutoff=f["pair_style"]["params"]["cutoff"], dt=d["params"]["dt"], units=s["units"],
            velocities=np.asarray(s["velocities"]), masses=np.asarray(s["masses"]),
            tags=np.asarray(s["tags"]), molecule_ids=np.asarray(s["molecule_ids"]),
            images=np.asarray(s["images"]),
            shift=bool(f["pair_style"]["params"].get("shift", False)),
            bonds=recs(t["bonds"], ("tag_i", "tag_j", "type")),
            angles=recs(t["angles"], ("tag_i", "tag_j", "tag_k", "type")),
            dihedrals=recs(t["dihedrals"], ("tag_i", "tag_j", "tag_k", "tag_l", "type")),
            bond_k=coeffs("bond", "k"), bond_r0=coeffs("bond", "r0"),
            angle_k=coeffs("angle", "k"), angle_theta0=coeffs("angle", "theta0"),
            dihedral_k=coeffs("dihedral", "k"), dihedral_d=coeffs("dihedral", "d"),
            dihedral_n=coeffs("dihedral", "n"),
            exclusion_distance=f.get("bonded_exclusion_distance") or 0,
            cutoff_buffer=nb["cutoff_buffer"], rebuild_check_every=nb["rebuild_check_every"],
            sort_every_rebuild=nb["sort_every_rebuild"], max_neighbors=nb["max_neighbors"],
            thermostat=None if thermo is None else (thermo["params"]["temperature"],
                                                    thermo["params"]["tau"]))


def _descriptors(spec: ReplicaSpec, keep: _lib.Keep):
    sd = _lib.SystemDesc()
    n = spec.n
    sd.n_particles = n
    if spec.units not in _lib.UNITS:
        raise ValueError('system.units must be "reduced" or "nm_kjmol".')
    sd.units = _lib.UNITS[spec.units]
    bb = np.asarray(spec.box_bound, dtype=np.float32).reshape(2, 3)
    sd.box_lo[:] = [float(x) for x in bb[0]]
    sd.box_hi[:] = [float(x) for x in bb[1]]
    sd.positions = keep.ptr(spec.positions, np.float32, ctypes.c_float)
    sd.velocities = keep.ptr(spec.velocities, np.float32, ctypes.c_float)
    sd.masses = keep.ptr(spec.masses, np.float32, ctypes.c_float)
    sd.types = keep.ptr(spec.types, np.int32, ctypes.c_int32)
    sd.tags = keep.ptr(spec.tags, np.uint32, ctypes.c_uint32)
    sd.molecule_ids = keep.ptr(spec.molecule_ids, np.uint32, ctypes.c_uint32)
    sd.images = keep.ptr(spec.images, np.int32, ctypes.c_int32)
    for name, width in (("bonds", 3), ("angles", 4), ("dihedrals", 5)):
        rec = getattr(spec, name)
        count = 0 if rec is None else int(np.asarray(rec).reshape(-1, width).shape[0])
        setattr(sd, "n_" + name, count)
        setattr(sd, name, keep.ptr(None if count == 0 else rec, np.uint32, ctypes.c_uint32))

    fd = _lib.ForceFieldDesc()
    eps = np.asarray(spec.epsilon, dtype=np.float64)
    fd.n_types = int(round(np.sqrt(eps.size)))
    fd.lj_epsilon = keep.ptr(eps, np.float64, ctypes.c_double)
    fd.lj_sigma = keep.ptr(spec.sigma, np.float64, ctypes.c_double)
    fd.lj_cutoff = float(spec.cutoff)
    fd.lj_shift = int(bool(spec.shift))
    fd.n_bond_types = 0 if spec.bond_k is None else len(spec.bond_k)
    fd.bond_k = keep.ptr(spec.bond_k, np.float64, ctypes.c_double)
    fd.bond_r0 = keep.ptr(spec.bond_r0, np.float64, ctypes.c_double)
    fd.n_angle_types = 0 if spec.angle_k is None else len(spec.angle_k)
    fd.angle_k = keep.ptr(spec.angle_k, np.float64, ctypes.c_double)
    fd.angle_theta0_deg = keep.ptr(spec.angle_theta0, np.float64, ctypes.c_double)
    fd.n_dihedral_types = 0 if spec.dihedral_k is None else len(spec.dihedral_k)
    fd.dihedral_k = keep.ptr(spec.dihedral_k, np.float64, ctypes.c_double)
    fd.dihedral_d = keep.ptr(spec.dihedral_d, np.int32, ctypes.c_int32)
    fd.dihedral_n = keep.ptr(spec.dihedral_n, np.int32, ctypes.c_int32)
    fd.exclusion_distance = int(spec.exclusion_distance)

    nd = _lib.NeighborDesc()
    nd.cutoff_buffer = float(spec.cutoff_buffer)
    nd.rebuild_check_every = int(spec.rebuild_check_every)
    nd.sort_every_rebuild = int(spec.sort_every_rebuild)
    nd.max_neighbors = int(spec.max_neighbors)

    dd = _lib.DynamicsDesc()
    dd.dt = float(spec.dt)
    if spec.thermostat is None:
        dd.thermostat = 0
    else:
        dd.thermostat = 1
        dd.temperature = float(spec.thermostat[0])
        dd.tau = float(spec.thermostat[1])
    return sd, fd, nd, dd


class Engine:
    """A device batch of replicas (one replica = one simulation)."""

    def __init__(self, replicas: ReplicaSpec | Sequence[ReplicaSpec]):
        if isinstance(replicas, ReplicaSpec):
            replicas = [replicas]
        self.replicas = list(replicas)
        L = _lib.load()
        keep = _lib.Keep()
        n = len(self.replicas)
        systems = (_lib.SystemDesc * n)()
        ffs = (_lib.ForceFieldDesc * n)()
        nbrs = (_lib.NeighborDesc * n)()
        dyns = (_lib.DynamicsDesc * n)()
        for r, spec in enumerate(self.replicas):
            systems[r], ffs[r], nbrs[r], dyns[r] = _descriptors(spec, keep)
        handle = ctypes.c_void_p()
        _lib.check(L.beads_batch_create(n, systems, ffs, nbrs, dyns, ctypes.byref(handle)))
        self._h = handle
        self._lib = L
        self.sizes = [spec.n for spec in self.replicas]
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)]).astype(np.int64)
        self.step = 0

    # -- lifetime ---------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.beads_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- stepping ---------------------------------------------------------
    def eval(self) -> list[dict]:
        out = (_lib.Observables * len(self.replicas))()
        _lib.check(self._lib.beads_eval(self._h, out))
        return [o.as_dict() for o in out]

    def run(self, steps: int, obs_every: int = 0) -> list[dict] | None:
        out = (_lib.Observables * len(self.replicas))()
        _lib.check(self._lib.beads_run(self._h, int(steps), int(obs_every), out))
        self.step += int(steps)
        if obs_every and steps and self.step % int(obs_every) == 0:
            return [o.as_dict() for o in out]
        return None

    def minimize(self, iterations: int, dmax: float, fref: float) -> None:
        _lib.check(self._lib.beads_minimize(self._h, int(iterations), float(dmax), float(fref)))
        self.step = 0

    # -- state --------------------------------------------------------------
    def state(self, replica: int = 0) -> dict:
        n = self.sizes[replica]
        pos = np.zeros((n, 3), np.float32)
        vel = np.zeros((n, 3), np.float32)
        force = np.zeros((n, 3), np.float32)
        img = np.zeros((n, 3), np.int32)
        _lib.check(self._lib.beads_get_state(self._h, replica, pos.ctypes.data, vel.ctypes.data,
                                             force.ctypes.data, img.ctypes.data))
        return {"positions": pos, "velocities": vel, "forces": force, "images": img}

    def set_state(self, replica: int, positions=None, velocities=None) -> None:
        p = None if positions is None else np.ascontiguousarray(positions, np.float32)
        v = None if velocities is None else np.ascontiguousarray(velocities, np.float32)
        _lib.check(self._lib.beads_set_state(self._h, replica,
                                             None if p is None else p.ctypes.data,
                                             None if v is None else v.ctypes.data))

    def upload_all(self, positions=None, velocities=None) -> None:
        p = None if positions is None else np.ascontiguousarray(positions, np.float32)
        v = None if velocities is None else np.ascontiguousarray(velocities, np.float32)
        _lib.check(self._lib.beads_upload_all(self._h, None if p is None else p.ctypes.data,
                                              None if v is None else v.ctypes.data))

    def download_all(self, positions: np.ndarray, velocities: np.ndarray | None = None) -> None:
        _lib.check(self._lib.beads_download_all(
            self._h, positions.ctypes.data, None if velocities is None else velocities.ctypes.data))

    def info(self) -> dict:
        nr = ctypes.c_uint32()
        nt = ctypes.c_uint64()
        st = ctypes.c_void_p()
        _lib.check(self._lib.beads_ctx_info(self._h, ctypes.byref(nr), ctypes.byref(nt),
                                            ctypes.byref(st)))
        return {"n_replicas": nr.value, "n_particles": nt.value, "stream": st.value or 0}

    def profile(self, stage: str, reps: int) -> float:
        """Mean milliseconds per launch of 'forces', 'step', 'rebuild',
        'forces_kick' (the force kernel as a step runs it, with the second
        half-kick; velocities and step state are restored afterwards), 'pair'
        (the pair-force kernel alone) or 'bonded' (the bonded kernel alone)."""
        code = {"forces": 0, "step": 1, "rebuild": 2, "forces_kick": 3, "pair": 4,
                "bonded": 5}[stage]
        out = ctypes.c_double()
        _lib.check(self._lib.beads_profile(self._h, code, int(reps), ctypes.byref(out)))
        if code == 1:
            self.step += int(reps)
        return out.value

    def set_tuning(self, threads_per_particle: int = 0, fuse_post: bool = False,
                   batch_depth: int = 8, list_bypass_l1: bool = False) -> None:
        """Fix the kernel schedule (threads per particle 1, 2 or 4; fused
        second half-kick; list entries in flight 4 or 8; list loads that
        bypass L1), or hand it back to the autotuner with
        threads_per_particle 0."""
        sched = (ctypes.c_int32 * 4)(int(threads_per_particle), 1 if fuse_post else 0,
                                     int(batch_depth), 1 if list_bypass_l1 else 0)
        _lib.check(self._lib.beads_set_tuning(self._h, sched))

    def tuning(self) -> dict:
        """The kernel schedule; "staged" is the list layout (not part of
        set_tuning: see set_list_staged)."""
        out = (ctypes.c_int32 * 5)()
        _lib.check(self._lib.beads_get_tuning(self._h, out))
        return {"threads_per_particle": out[0], "fuse_post": bool(out[1]),
                "batch_depth": out[2], "list_bypass_l1": bool(out[3]),
                "autotuned": bool(out[4]), "staged": self.list_staged()}

    def set_list_staged(self, staged: bool) -> None:
        """Pair forces from shared-memory cell tiles (True) or global gathers
        (False); the same bits either way (beads_set_list_layout).  Once set,
        the autotuner keeps this layout instead of timing both."""
        _lib.check(self._lib.beads_set_list_layout(self._h, 1 if staged else 0))

    def list_staged(self) -> bool:
        out = ctypes.c_int32()
        _lib.check(self._lib.beads_get_list_layout(self._h, ctypes.byref(out)))
        return bool(out.value)

    # -- differentiation ------------------------------------------------------
    def set_lj(self, replica: int, epsilon, sigma) -> None:
        """Replace one replica's LJ tables (symmetric n_types x n_types)."""
        eps = np.ascontiguousarray(epsilon, dtype=np.float64)
        sig = np.ascontiguousarray(sigma, dtype=np.float64)
        nt = len(self.replicas[replica].epsilon)
        if eps.shape != (nt, nt) or sig.shape != (nt, nt):
            raise ValueError(f"LJ tables of replica {replica} must be {nt} x {nt}.")
        _lib.check(self._lib.beads_set_lj(self._h, int(replica), eps.ctypes.data,
                                          sig.ctypes.data))

    def set_bonded(self, replica: int, bond_k=None, bond_r0=None, angle_k=None,
                   angle_theta0=None, dihedral_k=None) -> None:
        """Replace one replica's harmonic bonded parameters (per local type;
        None leaves a parameter unchanged; theta0 in degrees)."""
        keep = []

        def ptr(x):
            if x is None:
                return None
            a = np.ascontiguousarray(x, dtype=np.float64).ravel()
            keep.append(a)
            return a.ctypes.data

        _lib.check(self._lib.beads_set_bonded(self._h, int(replica), ptr(bond_k), ptr(bond_r0),
                                              ptr(angle_k), ptr(angle_theta0), ptr(dihedral_k)))

    def adjoint_bonded_grads(self) -> dict:
        """Bonded parameter gradients of the last adjoint_backward, one row
        per replica type in batch order: bond (d/dk, d/dr0), angle (d/dk,
        d/dtheta0 per degree), dihedral (d/dk)."""
        def count(x):
            return 0 if x is None else len(x)

        nb = sum(count(s.bond_k) for s in self.replicas)
        na = sum(count(s.angle_k) for s in self.replicas)
        nd = sum(count(s.dihedral_k) for s in self.replicas)
        gb = np.zeros((nb, 2), np.float64)
        ga = np.zeros((na, 2), np.float64)
        gd = np.zeros(nd, np.float64)
        _lib.check(self._lib.beads_adjoint_bonded_grads(self._h, gb.ctypes.data, ga.ctypes.data,
                                                        gd.ctypes.data))
        return {"bond": gb, "angle": ga, "dihedral": gd}

    def adjoint_forward(self, steps: int, record_from: int, checkpoint_every: int) -> np.ndarray:
        """Run `steps` steps keeping checkpoints; returns [PE, virial, KE] of
        steps record_from..steps, shape (steps - record_from + 1, R, 3)."""
        out = np.zeros((int(steps) - int(record_from) + 1, len(self.replicas), 3), np.float64)
        _lib.check(self._lib.beads_adjoint_forward(self._h, int(steps), int(record_from),
                                                   int(checkpoint_every), out.ctypes.data))
        self.step += int(steps)
        self._adjoint_shape = out.shape
        return out

    def adjoint_backward(self, obs_grad) -> tuple[list, list, np.ndarray, np.ndarray]:
        """dL/d(eps), dL/d(sigma) (one n_types x n_types array per replica,
        per ordered type pair) and dL/d(x0), dL/d(v0) (tag order) for the
        last adjoint_forward, given dL/d(observables)."""
        g = np.ascontiguousarray(obs_grad, dtype=np.float64)
        if g.shape != getattr(self, "_adjoint_shape", None):
            raise ValueError("observable gradient does not match the last adjoint_forward.")
        sizes = [len(spec.epsilon) for spec in self.replicas]
        n_par = sum(nt * nt for nt in sizes)
        ge = np.zeros(n_par, np.float64)
        gs = np.zeros(n_par, np.float64)
        gx = np.zeros((int(self.offsets[-1]), 3), np.float32)
        gv = np.zeros((int(self.offsets[-1]), 3), np.float32)
        _lib.check(self._lib.beads_adjoint_backward(self._h, g.ctypes.data, ge.ctypes.data,
                                                    gs.ctypes.data, gx.ctypes.data,
                                                    gv.ctypes.data))
        out_e, out_s, at = [], [], 0
        for nt in sizes:
            out_e.append(ge[at:at + nt * nt].reshape(nt, nt))
            out_s.append(gs[at:at + nt * nt].reshape(nt, nt))
            at += nt * nt
        return out_e, out_s, gx, gv

    def counters(self, replica: int = 0) -> dict:
        """Completed steps, neighbour builds and dangerous rebuilds of one
        replica; launches of the rebuild chain (whole batch)."""
        out = (ctypes.c_uint64 * 4)()
        _lib.check(self._lib.beads_counters(self._h, int(replica), out))
        return {"steps": int(out[0]), "builds": int(out[1]), "dangerous": int(out[2]),
                "chain_launches": int(out[3])}

    def launch_counts(self) -> dict:
        """Kernels per MD step and per rebuild chain under the current
        schedule (see beads_launch_counts); per_rebuild_chain is 0 when every
        step launches the chain."""
        per_step = ctypes.c_uint32()
        per_chain = ctypes.c_uint32()
        _lib.check(self._lib.beads_launch_counts(self._h, ctypes.byref(per_step),
                                                 ctypes.byref(per_chain)))
        return {"per_step": per_step.value, "per_rebuild_chain": per_chain.value}

    def list_stats(self) -> dict:
        total = ctypes.c_uint64()
        mx = ctypes.c_uint32()
        _lib.check(self._lib.beads_list_stats(self._h, ctypes.byref(total), ctypes.byref(mx)))
        return {"entries": total.value, "max": mx.value}

    # -- parity views ----------------------------------------------------------
    def debug_cells(self, replica: int = 0) -> np.ndarray:
        out = np.zeros(self.sizes[replica], np.uint32)
        _lib.check(self._lib.beads_debug_cells(self._h, replica, out.ctypes.data))
        return out

    def debug_neighbors(self, replica: int = 0, cap: int | None = None):
        cap = cap or int(self.replicas[replica].max_neighbors)
        n = self.sizes[replica]
        counts = np.zeros(n, np.uint32)
        partners = np.zeros((n, cap), np.uint32)
        _lib.check(self._lib.beads_debug_neighbors(self._h, replica, cap, counts.ctypes.data,
                                                   partners.ctypes.data))
        return counts, partners

    def debug_plan(self, replica: int = 0) -> dict:
        path = ctypes.c_int32()
        nc = np.zeros(3, np.uint32)
        _lib.check(self._lib.beads_debug_plan(self._h, replica, ctypes.byref(path), nc.ctypes.data))
        return {"path": ("direct", "regular_cell", "small_dimension")[path.value], "nc": nc}
