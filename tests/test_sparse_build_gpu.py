"""The two list-build forms against each other, on the GPU.

A replica whose cells hold few particles builds its lists one thread per
particle (k_build_sparse); the others a warp per cell (k_build).  Both walk
the same stencil segments in the same order with the same float expressions,
so the lists must be equal entry for entry, in order, and everything that
follows must be bit-identical: forces at step 0, and the whole state after a
run with rebuilds, reorders and the thermostat.  BEADS_BUILD forces one form
for every replica of the process (read when an engine is created).  Covered:
a bead-spring melt (exclusions, bonded terms; the sparse form's own case),
the LJ lattice and the binary mixture (dense by default), small-dimension
and direct grids, crowded cells, and a batch holding both kinds of replica,
in both list layouts.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

from beads_b200 import workloads
from beads_b200.engine import Engine
from tests.golden.make_reference_neighbor_fixtures import generated_case

pytestmark = pytest.mark.gpu

CASES = {
    "melt": lambda: [workloads.polymer_melt(n_chains=60, beads=50, seed=3, max_neighbors=96)],
    "lattice": lambda: [workloads.lj_lattice(n_side=12)],
    "mixture": lambda: [generated_case("mixture_64k")],
    "small_dim": lambda: [generated_case("small_dim")],
    "direct": lambda: [generated_case("direct")],
    "crowded": lambda: [generated_case("crowded")],
    "batch": lambda: [workloads.polymer_melt(n_chains=20, beads=50, seed=4, max_neighbors=96)]
    + workloads.replica_batch(3, n_min=256, n_max=4000, seed=5),
}


def _run(specs, form: str, staged: bool, steps: int):
    old = os.environ.get("BEADS_BUILD")
    os.environ["BEADS_BUILD"] = form
    try:
        eng = Engine(specs)
    finally:
        if old is None:
            del os.environ["BEADS_BUILD"]
        else:
            os.environ["BEADS_BUILD"] = old
    with eng:
        eng.set_list_staged(staged)
        try:
            eng.eval()
        except OverflowError:
            pass  # unrelaxed generated inputs: only the lists are compared then
        lists = [eng.debug_neighbors(r) for r in range(len(specs))]
        f0 = [eng.state(r)["forces"] for r in range(len(specs))]
        st = None
        if steps:
            eng.run(steps)
            st = [eng.state(r) for r in range(len(specs))]
            lists += [eng.debug_neighbors(r) for r in range(len(specs))]
    return lists, f0, st


@pytest.mark.parametrize("staged", [False, True], ids=["slot", "staged"])
@pytest.mark.parametrize("which", list(CASES))
def test_sparse_and_dense_builds_give_the_same_bits(which, staged):
    specs = CASES[which]()
    steps = 0 if which in ("mixture", "small_dim", "direct", "crowded") else 150
    a = _run(specs, "dense", staged, steps)
    b = _run(specs, "sparse", staged, steps)
    for (ca, pa), (cb, pb) in zip(a[0], b[0]):
        assert np.array_equal(ca, cb), which
        assert np.array_equal(pa, pb), which  # same entries in the same order
    for fa, fb in zip(a[1], b[1]):
        assert np.array_equal(fa, fb, equal_nan=True), which
    if steps:
        for sa, sb in zip(a[2], b[2]):
            for key in ("positions", "velocities", "forces", "images"):
                assert np.array_equal(sa[key], sb[key]), (which, key)
