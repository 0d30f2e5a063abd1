"""``ForceField``: pair style + coefficients, harmonic bonded styles, bonded
exclusions (the reference's python/beads/_forcefield.py contract)."""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Mapping

import numpy as np

from . import _checks as C

DEFAULT_EXCLUSION_DISTANCE = 2


@dataclass(frozen=True)
class StyleConfig:
    style: str
    params: Mapping[str, Any]


@dataclass(frozen=True)
class CoeffConfig:
    style: str
    key: tuple
    params: Mapping[str, Any]


@dataclass(frozen=True)
class ForceFieldConfig:
    pair_style: StyleConfig | None
    pair_coeffs: tuple[CoeffConfig, ...]
    bond_style: StyleConfig | None
    bond_coeffs: tuple[CoeffConfig, ...]
    angle_style: StyleConfig | None
    angle_coeffs: tuple[CoeffConfig, ...]
    dihedral_style: StyleConfig | None
    dihedral_coeffs: tuple[CoeffConfig, ...]
    bonded_exclusion_distance: int | None
    bonded_exclusion_policy: str


def _style_name(context: str, style) -> str:
    if not isinstance(style, str):
        raise TypeError(f"{context} name must be a string")
    if not style:
        raise ValueError(f"{context} name must not be empty")
    return style


class ForceField:
    """Builder for one pair style and optional harmonic bonded styles."""

    _KINDS = ("bond", "angle", "dihedral")

    def __init__(self) -> None:
        self._pair_style: tuple[str, dict] | None = None
        self._pair_coeffs: dict[tuple[int, int], tuple[str, dict]] = {}
        self._styles: dict[str, tuple[str, dict] | None] = {k: None for k in self._KINDS}
        self._coeffs: dict[str, dict[int, tuple[str, dict]]] = {k: {} for k in self._KINDS}
        self._exclusion_distance: int | None = None
        self._exclusion_policy: str | None = None
        self._frozen = False

    def _mutable(self) -> None:
        if self._frozen:
            raise RuntimeError("ForceField is frozen after binding to a Simulation.")

    # ---- pair -----------------------------------------------------------
    def pair_style(self, style: str, /, **params) -> "ForceField":
        self._mutable()
        if self._pair_style is not None:
            raise ValueError("ForceField supports one active pair_style.")
        self._pair_style = (_style_name("pair_style", style),
                            C.scalar_params("pair parameter", params, allow_bool=True))
        return self

    def pair_coeff(self, style: str, /, *, type_i, type_j, **params) -> "ForceField":
        self._mutable()
        if self._pair_style is None:
            raise ValueError("pair_style must be set before pair_coeff.")
        name = _style_name("pair_coeff style", style)
        if name != self._pair_style[0]:
            raise ValueError("pair_coeff style must match active pair_style.")
        a = C.positive_type("pair_coeff type_i", type_i)
        b = C.positive_type("pair_coeff type_j", type_j)
        key = (min(a, b), max(a, b))
        if key in self._pair_coeffs:
            raise ValueError(f"pair_coeff for types {key[0]} {key[1]} is already set.")
        self._pair_coeffs[key] = (name, C.scalar_params("pair parameter", params, allow_bool=True))
        return self

    # ---- bonded ---------------------------------------------------------
    def _set_style(self, kind: str, style, params) -> "ForceField":
        self._mutable()
        if self._styles[kind] is not None:
            raise ValueError(f"ForceField supports one active {kind}_style.")
        self._styles[kind] = (_style_name(f"{kind}_style", style),
                              C.scalar_params(f"{kind} parameter", params, allow_bool=True))
        return self

    def _set_coeff(self, kind: str, style, type_id, params) -> "ForceField":
        self._mutable()
        if self._styles[kind] is None:
            raise ValueError(f"{kind}_style must be set before {kind}_coeff.")
        name = _style_name(f"{kind}_coeff style", style)
        if name != self._styles[kind][0]:
            raise ValueError(f"{kind}_coeff style must match active {kind}_style.")
        t = C.positive_type(f"{kind}_coeff type", type_id)
        if t in self._coeffs[kind]:
            raise ValueError(f"{kind}_coeff for type {t} is already set.")
        self._coeffs[kind][t] = (name, C.scalar_params(f"{kind} parameter", params,
                                                        allow_bool=True))
        return self

    def bond_style(self, style: str, /, **params) -> "ForceField":
        return self._set_style("bond", style, params)

    def bond_coeff(self, style: str, /, *, type, **params) -> "ForceField":  # noqa: A002
        return self._set_coeff("bond", style, type, params)

    def angle_style(self, style: str, /, **params) -> "ForceField":
        return self._set_style("angle", style, params)

    def angle_coeff(self, style: str, /, *, type, **params) -> "ForceField":  # noqa: A002
        return self._set_coeff("angle", style, type, params)

    def dihedral_style(self, style: str, /, **params) -> "ForceField":
        return self._set_style("dihedral", style, params)

    def dihedral_coeff(self, style: str, /, *, type, **params) -> "ForceField":  # noqa: A002
        return self._set_coeff("dihedral", style, type, params)

    def exclude_bonded(self, *, distance=DEFAULT_EXCLUSION_DISTANCE) -> "ForceField":
        self._mutable()
        if self._exclusion_policy is not None:
            raise ValueError("ForceField bonded exclusions are already configured.")
        d = C.positive_int("bonded exclusion distance", distance)
        if d not in (1, 2, 3):
            raise ValueError("bonded exclusion distance must be 1, 2, or 3.")
        self._exclusion_distance = d
        self._exclusion_policy = "explicit"
        return self

    # ---- introspection (reference properties) -----------------------------
    @property
    def pair_style_name(self) -> str | None:
        return None if self._pair_style is None else self._pair_style[0]

    @property
    def pair_style_params(self) -> dict:
        return {} if self._pair_style is None else dict(self._pair_style[1])

    @property
    def pair_coeff_entries(self) -> tuple:
        return tuple((s, a, b, dict(p)) for (a, b), (s, p) in sorted(self._pair_coeffs.items()))

    # ---- freezing against a System ---------------------------------------
    def _freeze(self, system=None) -> ForceFieldConfig:
        distance = self._exclusion_distance
        policy = self._exclusion_policy
        if policy is None:
            if system is not None and system.topology.bonds:
                distance, policy = DEFAULT_EXCLUSION_DISTANCE, "default"
            else:
                policy = "none"

        def style(entry):
            return None if entry is None else StyleConfig(entry[0], C.frozen(entry[1]))

        cfg = ForceFieldConfig(
            pair_style=style(self._pair_style),
            pair_coeffs=tuple(CoeffConfig(s, k, C.frozen(p))
                              for k, (s, p) in sorted(self._pair_coeffs.items())),
            bond_style=style(self._styles["bond"]),
            bond_coeffs=tuple(CoeffConfig(s, (t,), C.frozen(p))
                              for t, (s, p) in sorted(self._coeffs["bond"].items())),
            angle_style=style(self._styles["angle"]),
            angle_coeffs=tuple(CoeffConfig(s, (t,), C.frozen(p))
                               for t, (s, p) in sorted(self._coeffs["angle"].items())),
            dihedral_style=style(self._styles["dihedral"]),
            dihedral_coeffs=tuple(CoeffConfig(s, (t,), C.frozen(p))
                                  for t, (s, p) in sorted(self._coeffs["dihedral"].items())),
            bonded_exclusion_distance=distance,
            bonded_exclusion_policy=policy,
        )
        if system is not None:
            _check_pair_coverage(cfg, system)
            topo = system.topology
            _check_bonded_coverage("bond", cfg.bond_style, cfg.bond_coeffs,
                                   {r[2] for r in topo.bonds}, bool(topo.bonds))
            _check_bonded_coverage("angle", cfg.angle_style, cfg.angle_coeffs,
                                   {r[3] for r in topo.angles}, bool(topo.angles))
            _check_bonded_coverage("dihedral", cfg.dihedral_style, cfg.dihedral_coeffs,
                                   {r[4] for r in topo.dihedrals}, bool(topo.dihedrals))
            if cfg.bonded_exclusion_distance is not None and not topo.bonds:
                raise ValueError("ForceField.exclude_bonded(...) requires System topology bonds.")
        self._frozen = True
        return cfg


def _check_pair_coverage(cfg: ForceFieldConfig, system) -> None:
    if cfg.pair_style is None:
        raise ValueError("ForceField requires an active pair_style.")
    active = sorted(int(t) for t in np.unique(system.types))
    expected = {(a, b) for a in active for b in active if a <= b}
    observed = {c.key for c in cfg.pair_coeffs}
    outside = sorted(k for k in observed if k[0] not in active or k[1] not in active)
    if outside:
        raise ValueError(
            f"ForceField pair_coeff type ids must be active System types; got {outside}.")
    missing = sorted(expected - observed)
    if missing:
        raise ValueError(
            f"ForceField pair_coeffs must cover all active System type pairs; missing {missing}.")


def _check_bonded_coverage(kind, style, coeffs, active_types, has_records) -> None:
    if style is None:
        if has_records:
            raise ValueError(f"System topology {kind}s require an active {kind}_style.")
        if coeffs:
            raise ValueError(f"{kind}_coeff requires an active {kind}_style.")
        return
    if not has_records:
        raise ValueError(f"{kind}_style requires System topology {kind}s.")
    observed = {c.key[0] for c in coeffs}
    missing = sorted(active_types - observed)
    if missing:
        raise ValueError(
            f"{kind}_coeffs must cover all active {kind} topology types; missing {missing}.")
    extra = sorted(observed - active_types)
    if extra:
        raise ValueError(f"{kind}_coeff types must be active {kind} topology types; got {extra}.")
