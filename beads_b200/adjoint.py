"""Differentiable MD trajectories.

``trajectory_observables`` runs a batch of replicas for a number of
velocity-Verlet steps and returns, per recorded step and replica, the
potential energy, the virial (sum r.F) and the kinetic energy as a torch
tensor that autograd can differentiate with respect to the LJ epsilon and
sigma tables, the initial positions and the initial velocities.  The
gradient is the engine's hand-written adjoint (beads_adjoint_forward /
beads_adjoint_backward in include/beads_b200.h): checkpoints every
``checkpoint_every`` steps, each segment replayed with the neighbour list of
every forward step frozen, LJ force Jacobian-vector products and parameter
derivatives on the device.  A loss such as the squared deviation of the mean
potential energy and pressure from targets is then ordinary torch code on the
returned tensor (pressure = s (2 KE + W) / (3 V)).
"""

from __future__ import annotations

import numpy as np
import torch

from .engine import Engine

__all__ = ["trajectory_observables"]


class _TrajectoryFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, epsilon, sigma, positions, velocities, engine, steps, record_from, every):
        n_rep = len(engine.replicas)
        eps = epsilon.detach().to(torch.float64).cpu().numpy()
        sig = sigma.detach().to(torch.float64).cpu().numpy()
        shared = eps.ndim == 2
        for r in range(n_rep):
            engine.set_lj(r, eps if shared else eps[r], sig if shared else sig[r])
        pos = positions.detach().to(torch.float32).cpu().contiguous().numpy()
        vel = velocities.detach().to(torch.float32).cpu().contiguous().numpy()
        engine.upload_all(pos, vel)
        obs = engine.adjoint_forward(steps, record_from, every)
        ctx.engine = engine
        ctx.shared = shared
        ctx.param_dtype = epsilon.dtype
        ctx.x_dtype = positions.dtype
        ctx.v_dtype = velocities.dtype
        return torch.from_numpy(obs)

    @staticmethod
    def backward(ctx, grad):
        g = grad.detach().to(torch.float64).cpu().contiguous().numpy()
        ge, gs, gx, gv = ctx.engine.adjoint_backward(g)
        if ctx.shared:
            d_eps = torch.from_numpy(np.sum(ge, axis=0))
            d_sig = torch.from_numpy(np.sum(gs, axis=0))
        else:
            d_eps = torch.from_numpy(np.stack(ge))
            d_sig = torch.from_numpy(np.stack(gs))
        return (d_eps.to(ctx.param_dtype), d_sig.to(ctx.param_dtype),
                torch.from_numpy(gx).to(ctx.x_dtype), torch.from_numpy(gv).to(ctx.v_dtype),
                None, None, None, None)


def trajectory_observables(engine: Engine, epsilon: torch.Tensor, sigma: torch.Tensor,
                           positions: torch.Tensor, velocities: torch.Tensor, *, steps: int,
                           record_from: int = 0, checkpoint_every: int = 50) -> torch.Tensor:
    """Observables [PE, virial, KE] of steps record_from..steps for every
    replica of `engine`, shape (steps - record_from + 1, R, 3), float64.

    epsilon, sigma: (n_types, n_types) tables shared by all replicas, or
    (R, n_types, n_types) per replica; symmetric.  positions, velocities:
    (N_total, 3) in tag order, replicas concatenated in batch order.  The
    engine must hold a pair-only (LJ) batch with at most 4 particle types.
    """
    return _TrajectoryFunction.apply(epsilon, sigma, positions, velocities, engine, int(steps),
                                     int(record_from), int(checkpoint_every))
