"""Plain PyTorch FP64 restatement of the engine's discrete dynamics, for
checking the adjoint: all-pairs minimum image, LJ with cutoff (and energy
shift), velocity Verlet with the Berendsen scale applied at the next step's
pre-kick, observables [PE, virial, KE = lambda^2 K].  Autograd through it is
the FP64 reference gradient."""

from __future__ import annotations

import torch


def lj_terms(x, types, box, eps, sig, rc, shift):
    d = x[:, None, :] - x[None, :, :]
    d = d - box * torch.round(d / box)
    r2 = (d * d).sum(-1)
    n = x.shape[0]
    mask = (r2 < rc * rc) & ~torch.eye(n, dtype=torch.bool)
    r2s = torch.where(mask, r2, torch.ones_like(r2))
    e = eps[types][:, types]
    s = sig[types][:, types]
    inv = 1.0 / r2s
    sr6 = (s * s * inv) ** 3
    sr12 = sr6 * sr6
    phi = torch.where(mask, 24.0 * e * inv * (2.0 * sr12 - sr6), torch.zeros_like(r2))
    force = (phi[..., None] * d).sum(1)
    u = 4.0 * e * (sr12 - sr6)
    if shift:
        sc6 = (s * s / (rc * rc)) ** 3
        u = u - 4.0 * e * (sc6 * sc6 - sc6)
    pe = 0.5 * torch.where(mask, u, torch.zeros_like(u)).sum()
    w = 0.5 * (phi * r2s).sum()
    return force, pe, w


def trajectory(x0, v0, masses, types, box, eps, sig, rc, shift, dt, steps, record_from,
               thermostat=None):
    """Observables of steps record_from..steps, shape (T', 3)."""
    m = masses[:, None]
    h = 0.5 * dt
    n = x0.shape[0]
    dof = 3.0 * n - 3.0
    x, v = x0, v0
    lam = torch.ones((), dtype=x0.dtype)
    f, pe, w = lj_terms(x, types, box, eps, sig, rc, shift)
    kin = 0.5 * (m * v * v).sum()
    rows = []
    if record_from == 0:
        rows.append(torch.stack([pe, w, kin]))
    for step in range(1, steps + 1):
        u = lam * v + h * f / m
        x = x + dt * u
        f, pe, w = lj_terms(x, types, box, eps, sig, rc, shift)
        v = u + h * f / m
        kin = 0.5 * (m * v * v).sum()
        if thermostat is not None:
            kt, tau = thermostat
            arg = 1.0 + (dt / tau) * (kt * dof / (2.0 * kin) - 1.0)
            lam = torch.sqrt(torch.clamp(arg, min=0.0))
        if step >= record_from:
            rows.append(torch.stack([pe, w, lam * lam * kin]))
    return torch.stack(rows)
