"""Whole-batch host transfers (beads_upload_all / beads_download_all): tag
order replica after replica, an exact round trip, and host buffers that the
caller may reuse as soon as the call returns, pinned ones included (their
copies are asynchronous on the engine stream until the call synchronises)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from beads_b200 import workloads
from beads_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _pinned(shape):
    return torch.empty(shape, dtype=torch.float32, pin_memory=True).numpy()


def test_upload_download_round_trip_with_reused_pinned_buffers():
    specs = [workloads.lj_lattice(n_side=10), workloads.lj_lattice(n_side=8)]
    n = sum(s.n for s in specs)
    rng = np.random.default_rng(11)
    with Engine(specs) as eng:
        eng.eval()
        pos = _pinned((n, 3))
        vel = _pinned((n, 3))
        eng.download_all(pos, vel)
        # tag order, replica after replica: the first replica's block is its
        # own state in tag order
        first = eng.state(0)
        assert np.array_equal(pos[:specs[0].n], first["positions"])
        assert np.array_equal(vel[:specs[0].n], first["velocities"])
        # new velocities and slightly moved positions (inside the boxes)
        want_pos = pos.copy()
        at = 0
        for s in specs:
            lo = np.asarray(s.box_bound[0], np.float32)
            hi = np.asarray(s.box_bound[1], np.float32)
            moved = pos[at:at + s.n] + rng.uniform(-0.01, 0.01, (s.n, 3)).astype(np.float32)
            want_pos[at:at + s.n] = np.clip(moved, lo + 0.05, hi - 0.05)
            at += s.n
        want_vel = rng.normal(size=(n, 3)).astype(np.float32)
        pos[:] = want_pos
        vel[:] = want_vel
        eng.upload_all(pos, vel)
        # the call has returned: overwriting the pinned buffers must not reach
        # the device
        pos[:] = np.float32(1e6)
        vel[:] = np.float32(-1e6)
        out_pos = _pinned((n, 3))
        out_vel = _pinned((n, 3))
        eng.download_all(out_pos, out_vel)
        assert np.array_equal(out_pos, want_pos)
        assert np.array_equal(out_vel, want_vel)
