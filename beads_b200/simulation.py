"""``Simulation``: binds System, ForceField and Dynamics with neighbour and
output settings and runs them (the reference's python/beads/_simulation.py,
_neighbor.py and _output.py contract).  ``execute()`` builds the same spec
dict the reference builds and hands it to ``beads_b200._native``."""

from __future__ import annotations

import os
from dataclasses import dataclass

from . import _checks as C
from .dynamics import Dynamics
from .forcefield import ForceField
from .system import System

TRAJECTORY_FIELDS = ("tag", "type", "position", "image", "velocity", "force")
TRAJECTORY_DEFAULT = ("tag", "type", "position", "image")


@dataclass(frozen=True)
class NeighborConfig:
    cutoff_buffer: float = 0.3
    rebuild_check_every: int = 1
    sort_every_rebuild: int = 10
    max_neighbors: int = 512

    def __post_init__(self) -> None:
        buf = C.nonnegative_real("neighbor cutoff_buffer", self.cutoff_buffer)
        check = C.positive_steps("neighbor rebuild_check_every", self.rebuild_check_every)
        sort = C.positive_steps("neighbor sort_every_rebuild", self.sort_every_rebuild)
        cap = C.positive_index("neighbor max_neighbors", self.max_neighbors)
        if buf == 0.0 and check != 1:
            raise ValueError("neighbor cutoff_buffer=0 requires rebuild_check_every=1")
        object.__setattr__(self, "cutoff_buffer", buf)
        object.__setattr__(self, "rebuild_check_every", check)
        object.__setattr__(self, "sort_every_rebuild", sort)
        object.__setattr__(self, "max_neighbors", cap)


def output_prefix(label: str, prefix) -> str:
    try:
        value = os.fspath(prefix)
    except TypeError as exc:
        raise TypeError(f"{label} prefix must be a string or path-like object") from exc
    if not isinstance(value, str):
        raise TypeError(f"{label} prefix must be a string or path-like object")
    if not value:
        raise ValueError(f"{label} prefix must not be empty")
    return value


def trajectory_fields(fields) -> tuple[str, ...]:
    if fields is None:
        return TRAJECTORY_DEFAULT
    if isinstance(fields, (str, bytes)):
        raise TypeError("trajectory fields must be an iterable of strings")
    try:
        values = tuple(fields)
    except TypeError as exc:
        raise TypeError("trajectory fields must be an iterable of strings") from exc
    if not values:
        raise ValueError("trajectory fields must not be empty")
    for f in values:
        if not isinstance(f, str):
            raise TypeError("trajectory fields must contain only strings")
        if f not in TRAJECTORY_FIELDS:
            raise ValueError(f"trajectory field {f!r} is not supported")
    if values[0] != "tag":
        raise ValueError("trajectory fields must include tag as the first field")
    if len(set(values)) != len(values):
        raise ValueError("trajectory fields must not contain duplicates")
    order = [TRAJECTORY_FIELDS.index(f) for f in values]
    if order != sorted(order):
        raise ValueError("trajectory fields must follow canonical order: "
                         "tag,type,position,image,velocity,force")
    return values


class Simulation:
    """One run: ``set_runsteps``, ``set_neighbor``, ``set_thermo``,
    ``set_trajectory``, ``save_final_state``, ``set_logging``, ``execute``."""

    def __init__(self, *, system: System, forcefield: ForceField, dynamics: Dynamics):
        if not isinstance(system, System):
            raise TypeError("Simulation requires a System.")
        if not isinstance(forcefield, ForceField):
            raise TypeError("Simulation requires a ForceField.")
        if not isinstance(dynamics, Dynamics):
            raise TypeError("Simulation requires a Dynamics.")
        self._system = system._freeze()
        self._ff = forcefield._freeze(system)
        self._dyn = dynamics._freeze()
        self._neighbor = NeighborConfig()
        self._thermo = None
        self._final = None
        self._trajectory = None
        self._log = {"echo": "screen"}
        self._runsteps = 0
        self._executed = False

    def _editable(self, action: str = "modified") -> None:
        if self._executed:
            if action == "execute":
                raise RuntimeError("Simulation.execute() cannot be called after execute(); "
                                   "create a new Simulation for another run.")
            raise RuntimeError("Simulation cannot be modified after execute(); "
                               "create a new Simulation for another run.")

    def set_runsteps(self, runsteps) -> "Simulation":
        self._editable()
        self._runsteps = C.nonnegative_steps("runsteps", runsteps)
        return self

    def set_neighbor(self, *, cutoff_buffer=0.3, rebuild_check_every=1, sort_every_rebuild=10,
                     max_neighbors=512) -> "Simulation":
        self._editable()
        self._neighbor = NeighborConfig(cutoff_buffer, rebuild_check_every, sort_every_rebuild,
                                        max_neighbors)
        return self

    def set_thermo(self, *, every, prefix) -> "Simulation":
        self._editable()
        self._thermo = {"every": C.positive_steps("thermo every", every),
                        "prefix": output_prefix("thermo", prefix)}
        return self

    def save_final_state(self, *, prefix) -> "Simulation":
        self._editable()
        self._final = {"prefix": output_prefix("final_state", prefix)}
        return self

    def set_trajectory(self, *, every, prefix, fields=None) -> "Simulation":
        self._editable()
        self._trajectory = {"every": C.positive_steps("trajectory every", every),
                            "prefix": output_prefix("trajectory", prefix),
                            "fields": list(trajectory_fields(fields))}
        return self

    def set_logging(self, *, echo="screen", prefix=None) -> "Simulation":
        self._editable()
        if not isinstance(echo, str):
            raise TypeError("logging echo must be a string")
        if echo not in ("screen", "log", "both", "none"):
            raise ValueError("logging echo must be one of 'screen', 'log', 'both', or 'none'")
        if echo in ("log", "both"):
            if prefix is None:
                raise ValueError(f"logging echo={echo!r} requires a prefix")
            self._log = {"echo": echo, "prefix": output_prefix("log", prefix)}
        else:
            if prefix is not None:
                raise ValueError(f"logging echo={echo!r} does not accept a prefix")
            self._log = {"echo": echo}
        return self

    def _native_spec(self) -> dict:
        s, ff, dyn, nb = self._system, self._ff, self._dyn, self._neighbor
        output: dict = {"log": dict(self._log)}
        if self._thermo is not None:
            output["thermo"] = dict(self._thermo)
        if self._final is not None:
            output["final_state"] = dict(self._final)
        if self._trajectory is not None:
            output["trajectory"] = dict(self._trajectory)

        def style(cfg):
            return None if cfg is None else {"style": cfg.style, "params": dict(cfg.params)}

        dynamics = {"style": dyn.style, "params": dict(dyn.params)}
        if dyn.thermostat is not None:
            dynamics["thermostat"] = {"style": dyn.thermostat.style,
                                      "params": dict(dyn.thermostat.params)}
        topo = s.topology
        return {
            "system": {
                "units": s.units, "n_particles": s.n_particles, "box_bound": s.box_bound,
                "positions": s.positions, "velocities": s.velocities, "masses": s.masses,
                "types": s.types, "tags": s.tags, "molecule_ids": s.molecule_ids,
                "images": s.images,
                "topology": {
                    "bonds": [{"tag_i": a, "tag_j": b, "type": t} for a, b, t in topo.bonds],
                    "angles": [{"tag_i": a, "tag_j": b, "tag_k": c, "type": t}
                               for a, b, c, t in topo.angles],
                    "dihedrals": [{"tag_i": a, "tag_j": b, "tag_k": c, "tag_l": d, "type": t}
                                  for a, b, c, d, t in topo.dihedrals],
                },
            },
            "forcefield": {
                "pair_style": style(ff.pair_style),
                "pair_coeffs": [{"style": c.style, "type_i": c.key[0], "type_j": c.key[1],
                                 "params": dict(c.params)} for c in ff.pair_coeffs],
                "bond_style": style(ff.bond_style),
                "bond_coeffs": [{"style": c.style, "type": c.key[0], "params": dict(c.params)}
                                for c in ff.bond_coeffs],
                "angle_style": style(ff.angle_style),
                "angle_coeffs": [{"style": c.style, "type": c.key[0], "params": dict(c.params)}
                                 for c in ff.angle_coeffs],
                "dihedral_style": style(ff.dihedral_style),
                "dihedral_coeffs": [{"style": c.style, "type": c.key[0],
                                     "params": dict(c.params)} for c in ff.dihedral_coeffs],
                "bonded_exclusion_distance": ff.bonded_exclusion_distance,
                "bonded_exclusion_policy": ff.bonded_exclusion_policy,
            },
            "dynamics": dynamics,
            "neighbor": {"cutoff_buffer": nb.cutoff_buffer,
                         "rebuild_check_every": nb.rebuild_check_every,
                         "sort_every_rebuild": nb.sort_every_rebuild,
                         "max_neighbors": nb.max_neighbors},
            "output": output,
            "runsteps": self._runsteps,
        }

    def execute(self) -> None:
        self._editable("execute")
        self._executed = True
        from . import _native

        _native.execute_simulation(self._native_spec())
