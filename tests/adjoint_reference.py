"""Plain PyTorch FP64 restatement of the engine's discrete dynamics, for
checking the adjoint: all-pairs minimum image, LJ with cutoff (and energy
shift), velocity Verlet with the Berendsen scale applied at the next step's
pre-kick, observables [PE, virial, KE = lambda^2 K].  Autograd through it is
the FP64 reference gradient."""

from __future__ import annotations

import torch


def lj_terms(x, types, box, eps, sig, rc, shift, excluded=None):
    d = x[:, None, :] - x[None, :, :]
    d = d - box * torch.round(d / box)
    r2 = (d * d).sum(-1)
    n = x.shape[0]
    mask = (r2 < rc * rc) & ~torch.eye(n, dtype=torch.bool)
    if excluded is not None:
        mask = mask & ~excluded
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


def _arm(x, a, b, box):
    d = x[a] - x[b]
    return d - box * torch.round(d / box)


def bonded_terms(x, box, top, params):
    """Harmonic bond / angle / dihedral energy (the reference's conventions,
    theta0 in degrees, signed dihedral angle), forces -grad U and virial
    sum over terms of arm . F, all differentiable.  top: 0-based index arrays
    {"bonds": (nb, 3), "angles": (na, 4), "dihedrals": (nd, 5)} with the type
    in the last column; params: {"bond_k", "bond_r0", "angle_k",
    "angle_theta0", "dihedral_k", "dihedral_d", "dihedral_n"}."""
    energy = torch.zeros((), dtype=x.dtype)
    arms = []
    if top.get("bonds") is not None and len(top["bonds"]):
        b = top["bonds"]
        d = _arm(x, b[:, 0], b[:, 1], box)
        arms.append(d)
        r = torch.sqrt((d * d).sum(-1))
        energy = energy + (0.5 * params["bond_k"][b[:, 2]] * (r - params["bond_r0"][b[:, 2]]) ** 2).sum()
    if top.get("angles") is not None and len(top["angles"]):
        a = top["angles"]
        a1 = _arm(x, a[:, 0], a[:, 1], box)
        a2 = _arm(x, a[:, 2], a[:, 1], box)
        arms += [a1, a2]
        cs = (a1 * a2).sum(-1) / torch.sqrt((a1 * a1).sum(-1) * (a2 * a2).sum(-1))
        th = torch.acos(torch.clamp(cs, -1.0, 1.0))
        th0 = params["angle_theta0"][a[:, 3]] * (torch.pi / 180.0)
        energy = energy + (0.5 * params["angle_k"][a[:, 3]] * (th - th0) ** 2).sum()
    if top.get("dihedrals") is not None and len(top["dihedrals"]):
        q = top["dihedrals"]
        b0 = _arm(x, q[:, 0], q[:, 1], box)
        b1 = _arm(x, q[:, 2], q[:, 1], box)
        b2 = _arm(x, q[:, 2], q[:, 3], box)
        arms += [b0, b1, b2]
        m = torch.cross(b0, b1, dim=-1)
        nn = torch.cross(b1, b2, dim=-1)
        cs = (m * nn).sum(-1) / torch.sqrt((m * m).sum(-1) * (nn * nn).sum(-1))
        phi = torch.acos(torch.clamp(cs, -1.0, 1.0))
        phi = torch.where((b0 * nn).sum(-1) < 0.0, -phi, phi)
        t = q[:, 4]
        energy = energy + (params["dihedral_k"][t] *
                           (1.0 + params["dihedral_d"][t] * torch.cos(params["dihedral_n"][t] * phi))).sum()
    g_x, *g_arms = torch.autograd.grad(energy, [x] + arms, create_graph=True)
    virial = -sum((a * g).sum() for a, g in zip(arms, g_arms)) if arms else energy * 0.0
    return -g_x, energy, virial


def trajectory(x0, v0, masses, types, box, eps, sig, rc, shift, dt, steps, record_from,
               thermostat=None, excluded=None, top=None, params=None):
    """Observables of steps record_from..steps, shape (T', 3)."""
    m = masses[:, None]
    h = 0.5 * dt
    n = x0.shape[0]
    dof = 3.0 * n - 3.0
    x, v = x0, v0
    lam = torch.ones((), dtype=x0.dtype)

    def terms(x):
        f, pe, w = lj_terms(x, types, box, eps, sig, rc, shift, excluded)
        if top is not None:
            fb, eb, wb = bonded_terms(x, box, top, params)
            f, pe, w = f + fb, pe + eb, w + wb
        return f, pe, w

    f, pe, w = terms(x)
    kin = 0.5 * (m * v * v).sum()
    rows = []
    if record_from == 0:
        rows.append(torch.stack([pe, w, kin]))
    for step in range(1, steps + 1):
        u = lam * v + h * f / m
        x = x + dt * u
        f, pe, w = terms(x)
        v = u + h * f / m
        kin = 0.5 * (m * v * v).sum()
        if thermostat is not None:
            kt, tau = thermostat
            arg = 1.0 + (dt / tau) * (kt * dof / (2.0 * kin) - 1.0)
            lam = torch.sqrt(torch.clamp(arg, min=0.0))
        if step >= record_from:
            rows.append(torch.stack([pe, w, lam * lam * kin]))
    return torch.stack(rows)


def lj_pair_terms(x, types, box, eps, sig, rc, shift, pi, pj):
    """lj_terms over a fixed set of unordered pairs (pi < pj): every pair
    that can come within rc during the trajectory must be in the set.  As in
    lj_terms (and the full-list engine), the force on a particle uses its own
    row of the type tables, and the energy and virial take half of each
    ordered pair, so the table gradients split over [a, b] and [b, a] alike."""
    d = x[pi] - x[pj]
    d = d - box * torch.round(d / box)
    r2 = (d * d).sum(-1)
    mask = r2 < rc * rc
    r2s = torch.where(mask, r2, torch.ones_like(r2))
    inv = 1.0 / r2s
    ti, tj = types[pi], types[pj]

    def oriented(e, s):
        sr6 = (s * s * inv) ** 3
        sr12 = sr6 * sr6
        phi = torch.where(mask, 24.0 * e * inv * (2.0 * sr12 - sr6), torch.zeros_like(r2))
        u = 4.0 * e * (sr12 - sr6)
        if shift:
            sc6 = (s * s / (rc * rc)) ** 3
            u = u - 4.0 * e * (sc6 * sc6 - sc6)
        return phi, torch.where(mask, u, torch.zeros_like(u))

    phi_i, u_i = oriented(eps[ti, tj], sig[ti, tj])
    phi_j, u_j = oriented(eps[tj, ti], sig[tj, ti])
    force = (torch.zeros_like(x).index_add(0, pi, phi_i[:, None] * d)
             .index_add(0, pj, -phi_j[:, None] * d))
    pe = 0.5 * (u_i + u_j).sum()
    w = 0.5 * ((phi_i + phi_j) * r2s).sum()
    return force, pe, w


def trajectory_pairs(x0, v0, masses, types, box, eps, sig, rc, shift, dt, steps, record_from,
                     pi, pj, thermostat=None):
    """trajectory() with the pair terms over a fixed pair set (large systems).
    Returns the observables and the largest displacement of any particle from
    x0 over the run, which must stay below half the pair set's buffer."""
    m = masses[:, None]
    h = 0.5 * dt
    n = x0.shape[0]
    dof = 3.0 * n - 3.0
    x, v = x0, v0
    lam = torch.ones((), dtype=x0.dtype, device=x0.device)
    f, pe, w = lj_pair_terms(x, types, box, eps, sig, rc, shift, pi, pj)
    kin = 0.5 * (m * v * v).sum()
    rows = []
    moved = torch.zeros((), dtype=x0.dtype, device=x0.device)
    if record_from == 0:
        rows.append(torch.stack([pe, w, kin]))
    for step in range(1, steps + 1):
        u = lam * v + h * f / m
        x = x + dt * u
        moved = torch.maximum(moved, ((x - x0) ** 2).sum(-1).max().detach().sqrt())
        f, pe, w = lj_pair_terms(x, types, box, eps, sig, rc, shift, pi, pj)
        v = u + h * f / m
        kin = 0.5 * (m * v * v).sum()
        if thermostat is not None:
            kt, tau = thermostat
            arg = 1.0 + (dt / tau) * (kt * dof / (2.0 * kin) - 1.0)
            lam = torch.sqrt(torch.clamp(arg, min=0.0))
        if step >= record_from:
            rows.append(torch.stack([pe, w, lam * lam * kin]))
    return torch.stack(rows), float(moved)
