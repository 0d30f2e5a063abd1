"""Kernel launches per step and per rebuild chain, as the engine reports them
(beads_launch_counts: the kernel nodes of one captured step).  The bench's
gpu_launches figure is built from these counts."""

from __future__ import annotations

import pytest

from beads_b200 import workloads
from beads_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _counts(spec, fuse: bool):
    with Engine(spec) as eng:
        eng.set_tuning(2, fuse, 4, True)
        eng.set_list_staged(False)
        eng.run(5)
        return eng.launch_counts()


def test_lattice_step_and_chain_kernels():
    spec = workloads.lj_lattice(n_side=12)
    plain = _counts(spec, False)
    fused = _counts(spec, True)
    # pre, decide, pair forces, post, post finish; the fused schedule drops post
    assert plain["per_step"] == 5, plain
    assert fused["per_step"] == 4, fused
    # bin, scan (64 cells: one chunk, one scan kernel), scatter, cell sort,
    # two reorder kernels, build
    assert plain["per_rebuild_chain"] == 7, plain
    assert fused["per_rebuild_chain"] == 7, fused


def test_melt_adds_bonded_kernels_and_chain_stages():
    melt = workloads.polymer_melt(n_chains=20, beads=50, seed=4, max_neighbors=96)
    counts = _counts(melt, False)
    # bonded terms and their per-particle gather join the step
    assert counts["per_step"] == 7, counts
    # the sparse cell sort, the exclusion projection and the sparse build
    # (in place of the dense one) join the chain
    assert counts["per_rebuild_chain"] == 9, counts


def test_replicas_beyond_one_scan_chunk_take_the_three_kernel_scan():
    # A scan chunk holds 4,096 cells: a 46^3-site lattice (97,336 beads)
    # has 17^3 = 4,913 cells, two chunks.
    big = workloads.lj_lattice(n_side=46)
    counts = _counts(big, False)
    # bin, three scan kernels, scatter, cell sort, two reorder kernels, build
    assert counts["per_rebuild_chain"] == 9, counts
