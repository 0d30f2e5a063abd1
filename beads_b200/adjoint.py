"""Differentiable MD trajectories.

``trajectory_observables`` runs a batch of replicas for a number of
velocity-Verlet steps and returns, per recorded step and replica, the
potential energy, the virial (sum r.F) and the kinetic energy as a torch
tensor that autograd can differentiate with respect to the LJ epsilon and
sigma tables, the harmonic bond (k, r0), angle (k, theta0) and dihedral (k)
parameters, the initial positions and the initial velocities.  The gradient
is the engine's hand-written adjoint (beads_adjoint_forward /
beads_adjoint_backward in include/beads_b200.h): checkpoints every
``checkpoint_every`` steps, each segment replayed with the neighbour list of
every forward step frozen, LJ and bonded force Jacobian-vector products and
parameter derivatives on the device.  A loss such as the squared deviation of
the mean potential energy and pressure from targets is then ordinary torch
code on the returned tensor (pressure = s (2 KE + W) / (3 V)).
"""

from __future__ import annotations

import numpy as np
import torch

from .engine import Engine

__all__ = ["trajectory_observables"]

_BONDED = ("bond_k", "bond_r0", "angle_k", "angle_theta0", "dihedral_k")


class _TrajectoryFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, epsilon, sigma, positions, velocities, bond_k, bond_r0, angle_k,
                angle_theta0, dihedral_k, engine, steps, record_from, every):
        n_rep = len(engine.replicas)
        eps = epsilon.detach().to(torch.float64).cpu().numpy()
        sig = sigma.detach().to(torch.float64).cpu().numpy()
        shared = eps.ndim == 2
        bonded = [None if t is None else t.detach().to(torch.float64).cpu().numpy()
                  for t in (bond_k, bond_r0, angle_k, angle_theta0, dihedral_k)]
        for r in range(n_rep):
            engine.set_lj(r, eps if shared else eps[r], sig if shared else sig[r])
            if any(b is not None for b in bonded):
                engine.set_bonded(r, *bonded)
        pos = positions.detach().to(torch.float32).cpu().contiguous().numpy()
        vel = velocities.detach().to(torch.float32).cpu().contiguous().numpy()
        engine.upload_all(pos, vel)
        obs = engine.adjoint_forward(steps, record_from, every)
        ctx.engine = engine
        ctx.shared = shared
        ctx.dtypes = (epsilon.dtype, positions.dtype, velocities.dtype)
        ctx.bonded = [None if t is None else t.dtype for t in
                      (bond_k, bond_r0, angle_k, angle_theta0, dihedral_k)]
        return torch.from_numpy(obs)

    @staticmethod
    def backward(ctx, grad):
        g = grad.detach().to(torch.float64).cpu().contiguous().numpy()
        engine = ctx.engine
        ge, gs, gx, gv = engine.adjoint_backward(g)
        p_dtype, x_dtype, v_dtype = ctx.dtypes
        if ctx.shared:
            d_eps = torch.from_numpy(np.sum(ge, axis=0))
            d_sig = torch.from_numpy(np.sum(gs, axis=0))
        else:
            d_eps = torch.from_numpy(np.stack(ge))
            d_sig = torch.from_numpy(np.stack(gs))
        bonded_grads = [None] * 5
        if any(t is not None for t in ctx.bonded):
            # parameters shared by all replicas: sum the per-replica rows
            raw = engine.adjoint_bonded_grads()
            n_rep = len(engine.replicas)

            def per_type(rows):
                return rows.reshape(n_rep, -1, *rows.shape[1:]).sum(axis=0)

            b = per_type(raw["bond"]) if len(raw["bond"]) else None
            a = per_type(raw["angle"]) if len(raw["angle"]) else None
            d = per_type(raw["dihedral"]) if len(raw["dihedral"]) else None
            vals = [None if b is None else b[:, 0], None if b is None else b[:, 1],
                    None if a is None else a[:, 0], None if a is None else a[:, 1],
                    d]
            bonded_grads = [None if (t is None or val is None) else
                            torch.from_numpy(np.ascontiguousarray(val)).to(t)
                            for t, val in zip(ctx.bonded, vals)]
        return (d_eps.to(p_dtype), d_sig.to(p_dtype), torch.from_numpy(gx).to(x_dtype),
                torch.from_numpy(gv).to(v_dtype), *bonded_grads, None, None, None, None)


def trajectory_observables(engine: Engine, epsilon: torch.Tensor, sigma: torch.Tensor,
                           positions: torch.Tensor, velocities: torch.Tensor, *, steps: int,
                           record_from: int = 0, checkpoint_every: int = 50,
                           bond_k: torch.Tensor | None = None,
                           bond_r0: torch.Tensor | None = None,
                           angle_k: torch.Tensor | None = None,
                           angle_theta0: torch.Tensor | None = None,
                           dihedral_k: torch.Tensor | None = None) -> torch.Tensor:
    """Observables [PE, virial, KE] of steps record_from..steps for every
    replica of `engine`, shape (steps - record_from + 1, R, 3), float64.

    epsilon, sigma: (n_types, n_types) tables shared by all replicas, or
    (R, n_types, n_types) per replica; symmetric.  positions, velocities:
    (N_total, 3) in tag order, replicas concatenated in batch order.  Bonded
    parameters (optional, one value per bonded type, shared by all replicas;
    angle theta0 in degrees) replace the engine's and become differentiable.
    At most 4 particle types and 8 bonded types of each kind per replica.
    checkpoint_every = 0 keeps every step's state on the device (32 bytes per
    particle and step) instead of replaying segments in the backward pass.
    """
    return _TrajectoryFunction.apply(epsilon, sigma, positions, velocities, bond_k, bond_r0,
                                     angle_k, angle_theta0, dihedral_k, engine, int(steps),
                                     int(record_from), int(checkpoint_every))
