"""beads_cell_sort_static: the allocation-free cell sort, through the C ABI.

It serves callers that cannot call cudaMalloc (codes that own all device
memory in their own pool, or step loops that must not synchronize the device).
Its cell ids are compared bit for bit with those the engine reports through
beads_debug_cells for the same positions, on two calls in a row with
different systems (the second call also shows that the shared static counters
are cleared between calls); the sorted order is checked for being the stable
counting sort of those ids.  Grids the engine comparison does not reach are
checked against the oracle's cell ids (the reference's rule, clamps
included): crowded cells (~100 members, and more than the 8192 members the
block sort stages in shared memory), 2 cells per axis, and beads just
outside [lo, hi).
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from beads_b200 import _lib, workloads
from beads_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _static_sort(spec):
    import torch

    L = _lib.load()
    n = spec.n
    dev = torch.device("cuda", 0)
    pos = torch.from_numpy(np.ascontiguousarray(spec.positions, np.float32)).to(dev)
    cell_of = torch.zeros(n, dtype=torch.int32, device=dev)
    order = torch.zeros(n, dtype=torch.int32, device=dev)
    cap = 70000
    cell_start = torch.zeros(cap, dtype=torch.int32, device=dev)
    bb = np.asarray(spec.box_bound, np.float32).reshape(2, 3)
    lo = (ctypes.c_float * 3)(*bb[0].tolist())
    hi = (ctypes.c_float * 3)(*bb[1].tolist())
    n_cells = ctypes.c_uint32()
    stream = torch.cuda.current_stream(dev)
    _lib.check(L.beads_cell_sort_static(
        pos.data_ptr(), n, lo, hi, float(spec.cutoff), float(spec.cutoff_buffer),
        cell_of.data_ptr(), order.data_ptr(), cell_start.data_ptr(), cap,
        ctypes.byref(n_cells), ctypes.c_void_p(stream.cuda_stream)))
    stream.synchronize()
    nc = n_cells.value
    return (cell_of.cpu().numpy().view(np.uint32), order.cpu().numpy().view(np.uint32),
            cell_start.cpu().numpy().view(np.uint32)[: nc + 1], nc)


def _engine_cells(spec):
    with Engine(spec) as eng:
        eng.eval()
        return eng.debug_cells()


def _check_sorted(cell_of, order, cell_start, nc):
    n = cell_of.size
    assert np.array_equal(np.sort(order), np.arange(n))
    assert np.array_equal(cell_start, np.concatenate([[0], np.cumsum(np.bincount(cell_of, minlength=nc))]))
    for c in range(nc):
        members = order[cell_start[c]:cell_start[c + 1]]
        assert np.all(cell_of[members] == c)
        assert np.all(np.diff(members.astype(np.int64)) > 0)


def test_static_cell_sort_matches_engine_on_two_calls():
    # Two different grids (6^3 and 10^3 cells), both overlap-free so the
    # engine's evaluation stays in range.
    first = workloads.lj_lattice()
    second = workloads.lj_lattice(n_side=24, density=0.7, seed_pos=9)
    results = [_static_sort(first), _static_sort(second)]
    for spec, (cell_of, order, cell_start, nc) in zip((first, second), results):
        assert np.array_equal(cell_of, _engine_cells(spec))
        _check_sorted(cell_of, order, cell_start, nc)


def _uniform_spec(n, box, seed, cutoff=2.5, skin=0.3):
    spec = workloads.lj_lattice()
    rng = np.random.default_rng(seed)
    spec.positions = (rng.uniform(0.0, 1.0, (n, 3)) * np.asarray(box)).astype(np.float32)
    spec.box_bound = np.array([[0.0, 0.0, 0.0], box], np.float32)
    spec.cutoff, spec.cutoff_buffer = cutoff, skin
    return spec


@pytest.mark.parametrize("case", ["crowded_3", "two_cells", "outside", "huge_cells"])
def test_static_cell_sort_matches_oracle_on_edge_grids(oracle, case):
    if case == "crowded_3":
        spec = _uniform_spec(2700, (8.5, 8.5, 8.5), 3)      # 3^3 cells, ~100 per cell
    elif case == "two_cells":
        spec = _uniform_spec(500, (6.0, 6.0, 6.0), 4)       # 2^3 cells (direct grid)
    elif case == "outside":
        spec = _uniform_spec(3000, (12.0, 12.0, 12.0), 5)
        lo, hi = np.float32(0.0), np.float32(12.0)
        # beads just below lo and at or just above hi on each axis (clamped)
        spec.positions[:6, 0] = [np.nextafter(lo, np.float32(-1)), -1e-3, hi,
                                 np.nextafter(hi, np.float32(13)), 12.5, -0.7]
        spec.positions[6:12, 1] = spec.positions[:6, 0]
        spec.positions[12:18, 2] = spec.positions[:6, 0]
    else:
        spec = _uniform_spec(80000, (6.0, 6.0, 6.0), 6)     # 2^3 cells of ~10,000
    cell_of, order, cell_start, nc = _static_sort(spec)
    expect = oracle.cell_ids(spec.positions, spec.box_bound, spec.cutoff, spec.cutoff_buffer)
    assert np.array_equal(cell_of, expect)
    _check_sorted(cell_of, order, cell_start, nc)
    if case in ("crowded_3", "huge_cells"):
        assert np.diff(cell_start).max() > (8192 if case == "huge_cells" else 32)
    # a second call on the same input gives the same bits (counters cleared)
    again = _static_sort(spec)
    assert all(np.array_equal(a, b) for a, b in zip((cell_of, order, cell_start), again[:3]))


def test_static_cell_sort_rejects_grids_beyond_the_maximum():
    spec = workloads.lj_mixture(n=1000, box=80.0, seed=1)  # 80^3 cells > 65536
    with pytest.raises(ValueError, match="BEADS_STATIC_MAX_CELLS"):
        _static_sort(spec)
