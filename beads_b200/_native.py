"""Drop-in for the reference's ``beads._native`` module.

Two functions with the reference's contract (native/src/bindings/module.cpp:
15-55): ``build_info()`` and ``execute_simulation(spec)``.  The spec dict is
the one ``Simulation._native_spec()`` builds (python/beads/_simulation.py:
138-279); it is parsed here into the C-ABI descriptors of
include/beads_b200.h and run by ``beads_execute``, which writes the thermo
CSV, trajectory, final-state and log files.  Parse errors are ValueError /
TypeError as the reference's pybind11 layer raises them.
"""

from __future__ import annotations

import ctypes
from typing import Any, Mapping

import numpy as np

from . import _lib


def build_info() -> dict:
    return _lib.build_info()


# ---- spec parsing ----------------------------------------------------------

def _get(mapping: Mapping, key: str, path: str):
    if not isinstance(mapping, Mapping):
        raise TypeError(f"{path} must be a dict.")
    if key not in mapping:
        raise ValueError(f'{path} is missing required field "{key}".')
    return mapping[key]


def _uint(value, path: str) -> int:
    """Non-negative integer, refused as the reference's value reader does
    (native/src/bindings/native_spec_value_reader.hpp:18-44)."""
    if isinstance(value, (bool, np.bool_)) or not isinstance(value, (int, np.integer)):
        raise TypeError(f"{path} must be an integer.")
    if value < 0:
        raise ValueError(f"{path} must be non-negative.")
    if value > np.iinfo(np.uint64).max:
        raise ValueError(f"{path} contains values outside the supported uint64 range.")
    return int(value)


def _array(value, dtype, shape, path: str) -> np.ndarray:
    # Order and wording of native/src/bindings/ndarray_reader.hpp:38-72.
    if not isinstance(value, np.ndarray):
        raise TypeError(f"{path} must be a numpy array.")
    if value.dtype != np.dtype(dtype):
        raise TypeError(f"{path} must have dtype {np.dtype(dtype).name}.")
    if tuple(value.shape) != tuple(shape):
        raise ValueError(f"{path} must have shape {tuple(shape)}.")
    if not value.flags.c_contiguous:
        raise ValueError(f"{path} must be C-contiguous.")
    return value


def _real(params: Mapping, key: str, context: str, *, required=True, default=None,
          positive=False, nonnegative=False) -> float | None:
    if key not in params:
        if required:
            raise ValueError(f"{context}.{key} is required.")
        return default
    value = params[key]
    if isinstance(value, bool) or not isinstance(value, (int, float, np.integer, np.floating)):
        raise ValueError(f"{context}.{key} must be a real value.")
    out = float(value)
    if positive and not (np.isfinite(out) and out > 0.0):
        raise ValueError(f"{context}.{key} must be finite and positive.")
    if nonnegative and not (np.isfinite(out) and out >= 0.0):
        raise ValueError(f"{context}.{key} must be finite and non-negative.")
    return out


def _integer(params: Mapping, key: str, context: str) -> int:
    if key not in params:
        raise ValueError(f"{context}.{key} is required.")
    value = params[key]
    if isinstance(value, bool) or not isinstance(value, (int, np.integer)):
        raise ValueError(f"{context}.{key} must be an integer.")
    return int(value)


def _only(params: Mapping, allowed: set, context: str) -> None:
    for key in params:
        if key not in allowed:
            raise ValueError(f'{context} has unsupported parameter "{key}".')


def _exact(params: Mapping, keys: set, context: str) -> None:
    _only(params, keys, context)
    for key in keys:
        if key not in params:
            raise ValueError(f"{context}.{key} is required.")


def _style(entry, path: str, allowed: str, kind: str):
    if entry is None:
        return None
    style = _get(entry, "style", path)
    if style != allowed:
        raise ValueError(f'unsupported {kind} style "{style}".')
    return dict(_get(entry, "params", path))


class _Parsed:
    """Descriptors for one spec plus the NumPy buffers they point into."""

    def __init__(self, spec: Mapping[str, Any]):
        self.keep = _lib.Keep()
        system = _get(spec, "system", "native spec")
        ff = _get(spec, "forcefield", "native spec")
        dyn = _get(spec, "dynamics", "native spec")
        nbr = _get(spec, "neighbor", "native spec")
        out = _get(spec, "output", "native spec")
        self.runsteps = _uint(_get(spec, "runsteps", "native spec"), "runsteps")
        self._system(system)
        self._forcefield(ff)
        self._dynamics(dyn)
        self._neighbor(nbr)
        self._output(out)

    # system -------------------------------------------------------------
    def _system(self, s) -> None:
        units = _get(s, "units", "system")
        if units not in _lib.UNITS:
            raise ValueError('system.units must be "reduced" or "nm_kjmol".')
        n = int(_get(s, "n_particles", "system"))
        if n <= 0:
            raise ValueError("system.n_particles must be positive.")
        self.n = n
        box = _array(_get(s, "box_bound", "system"), np.float32, (2, 3), "system.box_bound")
        self.positions = _array(_get(s, "positions", "system"), np.float32, (n, 3),
                                "system.positions")
        vel = _array(_get(s, "velocities", "system"), np.float32, (n, 3), "system.velocities")
        masses = _array(_get(s, "masses", "system"), np.float32, (n,), "system.masses")
        self.types = _array(_get(s, "types", "system"), np.int32, (n,), "system.types")
        self.tags = _array(_get(s, "tags", "system"), np.uint32, (n,), "system.tags")
        mol = _array(_get(s, "molecule_ids", "system"), np.uint32, (n,), "system.molecule_ids")
        img = _array(_get(s, "images", "system"), np.int32, (n, 3), "system.images")
        topo = _get(s, "topology", "system")
        bonds = [(_get(b, "tag_i", "bond"), _get(b, "tag_j", "bond"), _get(b, "type", "bond"))
                 for b in _get(topo, "bonds", "system.topology")]
        angles = [tuple(_get(a, k, "angle") for k in ("tag_i", "tag_j", "tag_k", "type"))
                  for a in _get(topo, "angles", "system.topology")]
        dihs = [tuple(_get(d, k, "dihedral") for k in ("tag_i", "tag_j", "tag_k", "tag_l",
                                                       "type"))
                for d in _get(topo, "dihedrals", "system.topology")]
        sd = _lib.SystemDesc()
        sd.n_particles = n
        sd.units = _lib.UNITS[units]
        sd.box_lo[:] = [float(x) for x in box[0]]
        sd.box_hi[:] = [float(x) for x in box[1]]
        k = self.keep
        sd.positions = k.ptr(self.positions, np.float32, ctypes.c_float)
        sd.velocities = k.ptr(vel, np.float32, ctypes.c_float)
        sd.masses = k.ptr(masses, np.float32, ctypes.c_float)
        sd.types = k.ptr(self.types, np.int32, ctypes.c_int32)
        sd.tags = k.ptr(self.tags, np.uint32, ctypes.c_uint32)
        sd.molecule_ids = k.ptr(mol, np.uint32, ctypes.c_uint32)
        sd.images = k.ptr(img, np.int32, ctypes.c_int32)
        for name, recs, width in (("bonds", bonds, 3), ("angles", angles, 4),
                                  ("dihedrals", dihs, 5)):
            setattr(sd, "n_" + name, len(recs))
            arr = np.asarray(recs, dtype=np.int64).reshape(-1, width)
            if arr.size and (arr.min() < 0 or arr.max() > np.iinfo(np.uint32).max):
                raise ValueError(f"system.topology.{name} values are out of range.")
            setattr(sd, name, k.ptr(arr.astype(np.uint32) if len(recs) else None, np.uint32,
                                    ctypes.c_uint32))
        self.sd = sd
        self.n_types = int(self.types.max()) if n else 0
        self.bond_types = max((b[2] for b in bonds), default=0)
        self.angle_types = max((a[3] for a in angles), default=0)
        self.dihedral_types = max((d[4] for d in dihs), default=0)

    # force field ------------------------------------------------------------
    def _forcefield(self, f) -> None:
        pair = _get(f, "pair_style", "forcefield")
        if pair is None:
            raise ValueError("forcefield.pair_style is required.")
        pair_name = _get(pair, "style", "forcefield.pair_style")
        coeffs = _get(f, "pair_coeffs", "forcefield")
        # The style agreement is checked before the style itself is looked up
        # (native/src/input/native_spec_validation.hpp:484-488, then
        # native/src/forcefield/pair/pair_factory.cpp:44-46).
        for c in coeffs:
            if _get(c, "style", "pair_coeff") != pair_name:
                raise ValueError("forcefield.pair_coeff style must match active pair_style.")
        params = _style(pair, "forcefield.pair_style", "lj", "pair")
        _only(params, {"cutoff", "shift"}, 'Pair("lj") pair_style')
        cutoff = _real(params, "cutoff", 'Pair("lj") pair_style', positive=True)
        shift = params.get("shift", False)
        if not isinstance(shift, (bool, np.bool_)):
            raise ValueError('Pair("lj") pair_style.shift must be a boolean.')
        nt = self.n_types
        eps = np.full((nt, nt), np.nan)
        sig = np.full((nt, nt), np.nan)
        for c in coeffs:
            a, b = int(_get(c, "type_i", "pair_coeff")), int(_get(c, "type_j", "pair_coeff"))
            if not (1 <= a <= nt and 1 <= b <= nt):
                raise ValueError("Pair(\"lj\") pair_coeff type id is outside active type range.")
            p = dict(_get(c, "params", "pair_coeff"))
            _exact(p, {"epsilon", "sigma"}, 'Pair("lj") pair_coeff')
            e = _real(p, "epsilon", 'Pair("lj") pair_coeff', positive=True)
            s = _real(p, "sigma", 'Pair("lj") pair_coeff', positive=True)
            if not np.isnan(eps[a - 1, b - 1]):
                raise ValueError("Pair(\"lj\") pair_coeff duplicate coeff for type pair.")
            eps[a - 1, b - 1] = eps[b - 1, a - 1] = e
            sig[a - 1, b - 1] = sig[b - 1, a - 1] = s
        if np.isnan(eps).any():
            raise ValueError(
                "Pair(\"lj\") pair_coeff requires complete type-pair coeff coverage.")
        fd = _lib.ForceFieldDesc()
        k = self.keep
        fd.n_types = nt
        fd.lj_epsilon = k.ptr(eps, np.float64, ctypes.c_double)
        fd.lj_sigma = k.ptr(sig, np.float64, ctypes.c_double)
        fd.lj_cutoff = cutoff
        fd.lj_shift = int(bool(shift))
        self.cutoff = cutoff

        def table(kind, style_key, coeff_key, n_types, keys, label):
            style = _style(f.get(style_key), f"forcefield.{style_key}", "harmonic", kind)
            coeffs = f.get(coeff_key) or []
            if style is None:
                if n_types:
                    raise ValueError(f"System topology {kind}s require an active {kind}_style.")
                return None
            _exact(style, set(), f"{kind}_style")
            rows = [None] * n_types
            for c in coeffs:
                if _get(c, "style", f"{kind}_coeff") != "harmonic":
                    raise ValueError(f'unsupported {kind} style "{c["style"]}".')
                t = int(_get(c, "type", f"{kind}_coeff"))
                if not 1 <= t <= n_types:
                    raise ValueError(f'{label} {kind}_coeff type is not active in topology '
                                     f'{kind}s.')
                if rows[t - 1] is not None:
                    raise ValueError(f"{label} {kind}_coeffs must not contain duplicates.")
                p = dict(_get(c, "params", f"{kind}_coeff"))
                _exact(p, set(keys), f"{kind}_coeff")
                rows[t - 1] = p
            if any(r is None for r in rows):
                raise ValueError(f"{label} {kind}_coeffs must cover all active topology "
                                 f"{kind} types.")
            return rows

        bonds = table("bond", "bond_style", "bond_coeffs", self.bond_types, ("k", "r0"),
                      'Bond("harmonic")')
        angles = table("angle", "angle_style", "angle_coeffs", self.angle_types,
                       ("k", "theta0"), 'Angle("harmonic")')
        dihs = table("dihedral", "dihedral_style", "dihedral_coeffs", self.dihedral_types,
                     ("k", "d", "n"), 'Dihedral("harmonic")')
        if bonds:
            bk = [_real(r, "k", "bond_coeff", nonnegative=True) for r in bonds]
            br = [_real(r, "r0", "bond_coeff", nonnegative=True) for r in bonds]
            fd.n_bond_types = len(bonds)
            fd.bond_k = k.ptr(bk, np.float64, ctypes.c_double)
            fd.bond_r0 = k.ptr(br, np.float64, ctypes.c_double)
        if angles:
            ak = [_real(r, "k", "angle_coeff", nonnegative=True) for r in angles]
            at = [_real(r, "theta0", "angle_coeff", nonnegative=True) for r in angles]
            if any(t > 180.0 for t in at):
                raise ValueError('Angle("harmonic") angle_coeff.theta0 must be between 0 and '
                                 '180 degrees.')
            fd.n_angle_types = len(angles)
            fd.angle_k = k.ptr(ak, np.float64, ctypes.c_double)
            fd.angle_theta0_deg = k.ptr(at, np.float64, ctypes.c_double)
        if dihs:
            dk = [_real(r, "k", "dihedral_coeff", nonnegative=True) for r in dihs]
            dd = [_integer(r, "d", "dihedral_coeff") for r in dihs]
            dn = [_integer(r, "n", "dihedral_coeff") for r in dihs]
            if any(x not in (-1, 1) for x in dd):
                raise ValueError('Dihedral("harmonic") dihedral_coeff.d must be +1 or -1.')
            if any(x < 0 or x > np.iinfo(np.int32).max for x in dn):
                raise ValueError('Dihedral("harmonic") dihedral_coeff.n must be non-negative.')
            fd.n_dihedral_types = len(dihs)
            fd.dihedral_k = k.ptr(dk, np.float64, ctypes.c_double)
            fd.dihedral_d = k.ptr(dd, np.int32, ctypes.c_int32)
            fd.dihedral_n = k.ptr(dn, np.int32, ctypes.c_int32)
        dist = f.get("bonded_exclusion_distance")
        if dist is not None:
            dist = int(dist)
            if dist not in (1, 2, 3):
                raise ValueError("bonded exclusion distance must be 1, 2, or 3.")
        fd.exclusion_distance = 0 if dist is None else dist
        self.exclusion_policy = str(f.get("bonded_exclusion_policy", "none"))
        self.fd = fd

    # dynamics / neighbour / output ------------------------------------------------
    def _dynamics(self, d) -> None:
        if _get(d, "style", "dynamics") != "velocity_verlet":
            raise ValueError("dynamics.style must be velocity_verlet.")
        params = dict(_get(d, "params", "dynamics"))
        if set(params) != {"dt"}:
            raise ValueError('dynamics.params for style "velocity_verlet" requires exactly '
                             'parameter "dt".')
        dd = _lib.DynamicsDesc()
        dd.dt = _real(params, "dt", "dynamics.params", positive=True)
        thermo = d.get("thermostat")
        self.thermostat_name = "none"
        if thermo is not None:
            if _get(thermo, "style", "dynamics.thermostat") != "berendsen":
                raise ValueError("dynamics.thermostat.style supports only berendsen.")
            tp = dict(_get(thermo, "params", "dynamics.thermostat"))
            if set(tp) != {"temperature", "tau"}:
                raise ValueError('Thermostat("berendsen") requires exactly parameters '
                                 '"temperature" and "tau".')
            dd.thermostat = 1
            dd.temperature = _real(tp, "temperature", 'Thermostat("berendsen")',
                                   nonnegative=True)
            dd.tau = _real(tp, "tau", 'Thermostat("berendsen")', positive=True)
            self.thermostat_name = "berendsen"
        self.dd = dd

    def _neighbor(self, nb) -> None:
        # Checks and wording of native/src/input/native_spec_validation.hpp:649-669.
        nd = _lib.NeighborDesc()
        buffer = _real(nb, "cutoff_buffer", "neighbor")
        if not np.isfinite(buffer):
            raise ValueError("neighbor.cutoff_buffer must be finite.")
        if buffer < 0.0:
            raise ValueError("neighbor.cutoff_buffer must be non-negative.")
        counts = {}
        for key in ("rebuild_check_every", "sort_every_rebuild", "max_neighbors"):
            counts[key] = _uint(_get(nb, key, "neighbor"), f"neighbor.{key}")
            if counts[key] == 0:
                raise ValueError(f"neighbor.{key} must be positive.")
            if counts[key] > np.iinfo(np.uint32).max:
                raise ValueError(f"neighbor.{key} contains values outside the supported "
                                 "uint32 range.")
        if buffer == 0.0 and counts["rebuild_check_every"] != 1:
            raise ValueError("neighbor.cutoff_buffer=0 requires neighbor.rebuild_check_every=1.")
        nd.cutoff_buffer = buffer
        nd.rebuild_check_every = counts["rebuild_check_every"]
        nd.sort_every_rebuild = counts["sort_every_rebuild"]
        nd.max_neighbors = counts["max_neighbors"]
        self.nd = nd

    def _output(self, out) -> None:
        rd = _lib.RunDesc()
        rd.runsteps = self.runsteps
        self.strings: list[bytes] = []

        def text(value) -> bytes:
            b = str(value).encode()
            self.strings.append(b)
            return b

        thermo = out.get("thermo")
        if thermo is not None:
            rd.thermo_every = int(_get(thermo, "every", "output.thermo"))
            rd.thermo_prefix = text(_get(thermo, "prefix", "output.thermo"))
            if rd.thermo_every <= 0:
                raise ValueError("output.thermo.every must be positive.")
        traj = out.get("trajectory")
        if traj is not None:
            rd.trajectory_every = int(_get(traj, "every", "output.trajectory"))
            rd.trajectory_prefix = text(_get(traj, "prefix", "output.trajectory"))
            fields = list(_get(traj, "fields", "output.trajectory"))
            from .simulation import trajectory_fields

            try:
                trajectory_fields(fields)
            except (TypeError, ValueError) as exc:
                raise ValueError(f"output.trajectory.fields: {exc}") from exc
            rd.trajectory_fields = sum(_lib.FIELD_BITS[f] for f in fields)
            if rd.trajectory_every <= 0:
                raise ValueError("output.trajectory.every must be positive.")
        final = out.get("final_state")
        if final is not None:
            rd.final_state_prefix = text(_get(final, "prefix", "output.final_state"))
        log = out.get("log")
        echo = "none" if log is None else _get(log, "echo", "output.log")
        if echo not in _lib.ECHO:
            raise ValueError("output.log.echo must be screen, log, both, or none.")
        rd.log_echo = _lib.ECHO[echo]
        if log is not None and log.get("prefix") is not None:
            rd.log_prefix = text(log["prefix"])
        self.rd = rd


def execute_simulation(spec: Mapping[str, Any]) -> None:
    """Run one simulation spec; results are written to the requested files."""
    parsed = _Parsed(spec)
    L = _lib.load()
    rd = parsed.rd
    rd.system = ctypes.pointer(parsed.sd)
    rd.forcefield = ctypes.pointer(parsed.fd)
    rd.neighbor = ctypes.pointer(parsed.nd)
    rd.dynamics = ctypes.pointer(parsed.dd)
    rd.thermostat_name = parsed.thermostat_name.encode()
    rd.exclusion_policy = parsed.exclusion_policy.encode()
    interrupted = []

    def poll(_user) -> int:
        # The reference checks PyErr_CheckSignals between steps (module.cpp:29-34).
        try:
            if ctypes.pythonapi.PyErr_CheckSignals() != 0:
                interrupted.append(True)
                return 1
        except KeyboardInterrupt:
            interrupted.append(True)
            return 1
        return 0

    callback = _lib.INTERRUPT_FN(poll)
    rd.interrupt = callback
    status = L.beads_execute(ctypes.byref(rd))
    if status == _lib.ERR_INTERRUPTED or interrupted:
        raise KeyboardInterrupt
    _lib.check(status)
