"""``Dynamics``: velocity Verlet with an optional Berendsen thermostat (the
reference's python/beads/_dynamics.py contract)."""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Mapping

from . import _checks as C


@dataclass(frozen=True)
class ThermostatConfig:
    style: str
    params: Mapping[str, Any]


@dataclass(frozen=True)
class DynamicsConfig:
    style: str
    params: Mapping[str, Any]
    thermostat: ThermostatConfig | None = None


def _named(kind: str, style, allowed: str) -> str:
    if not isinstance(style, str):
        raise TypeError(f"{kind} style must be a string.")
    if not style:
        raise ValueError(f"{kind} style must not be empty.")
    if style != allowed:
        raise ValueError(f"Unknown {kind} style {style!r}.")
    return style


class Dynamics:
    """``Dynamics("velocity_verlet", dt=...)``; thermostat via
    ``set_thermostat("berendsen", temperature=..., tau=...)``."""

    def __init__(self, style: str, /, **params) -> None:
        self._style = _named("Dynamics", style, "velocity_verlet")
        self._params = C.scalar_params("Dynamics parameter", params, allow_bool=False)
        if set(self._params) != {"dt"}:
            raise ValueError('Dynamics("velocity_verlet") requires exactly parameter "dt".')
        dt = self._params["dt"]
        if not isinstance(dt, (int, float)) or dt <= 0:
            raise ValueError("Dynamics dt must be positive.")
        self._thermostat: ThermostatConfig | None = None
        self._frozen = False

    @property
    def style(self) -> str:
        return self._style

    @property
    def params(self) -> dict:
        return dict(self._params)

    def set_thermostat(self, style: str, /, **params) -> "Dynamics":
        if self._frozen:
            raise RuntimeError("Dynamics is frozen after binding to a Simulation.")
        name = _named("Thermostat", style, "berendsen")
        values = C.scalar_params("Thermostat parameter", params, allow_bool=False)
        if set(values) != {"temperature", "tau"}:
            raise ValueError('Thermostat("berendsen") requires exactly parameters '
                             '"temperature" and "tau".')
        for key in ("temperature", "tau"):
            if not isinstance(values[key], (int, float)):
                raise TypeError(f"Thermostat parameter {key} must be a real number.")
        if float(values["temperature"]) < 0.0:
            raise ValueError("Thermostat temperature must be non-negative.")
        if float(values["tau"]) <= 0.0:
            raise ValueError("Thermostat tau must be positive.")
        self._thermostat = ThermostatConfig(name, C.frozen(values))
        return self

    def _freeze(self) -> DynamicsConfig:
        self._frozen = True
        return DynamicsConfig(self._style, C.frozen(self._params), self._thermostat)
