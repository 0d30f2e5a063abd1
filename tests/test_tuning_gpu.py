"""Kernel schedules (threads per particle, fused or separate second
half-kick) never change a result, and the autotuner settles on one of them."""

from __future__ import annotations

import numpy as np
import pytest

from beads_b200 import workloads
from beads_b200.engine import Engine, ReplicaSpec
from tests.test_reference_pin import fixture

pytestmark = pytest.mark.gpu

SCHEDULES = [(tpa, fuse, depth, pf) for tpa in (1, 2, 4) for depth in (8, 4)
             for fuse in (False, True) for pf in (True, False)]


def _case(name):
    if name == "batch":
        return workloads.replica_batch(6, n_min=256, n_max=3000, seed=11)
    _, spec = fixture(name)
    return ReplicaSpec.from_spec(spec)


@pytest.mark.parametrize("name", ["mixture", "chains", "batch"])
def test_every_schedule_gives_identical_bits(name):
    spec = _case(name)
    outs = []
    runs = [(sched, staged) for sched in SCHEDULES for staged in (True, False)]
    for (tpa, fuse, depth, pf), staged in runs:
        with Engine(spec) as eng:
            eng.set_tuning(tpa, fuse, depth, pf)
            eng.set_list_staged(staged)
            rows = [eng.run(20, 20), eng.run(20, 20)]
            states = [eng.state(r) for r in range(len(eng.sizes))]
            t = eng.tuning()
            got = t.pop("staged")
            assert got == staged or (name == "batch" and not got)
            assert t == {"threads_per_particle": tpa, "fuse_post": fuse,
                         "batch_depth": depth, "list_bypass_l1": pf, "autotuned": False}
        outs.append((rows, states))
    rows0, states0 = outs[0]
    for (rows, states), sched in zip(outs[1:], runs[1:]):
        assert rows == rows0, sched
        for a, b in zip(states, states0):
            for key in ("positions", "velocities", "forces", "images"):
                assert np.array_equal(a[key], b[key]), (sched, key)


def test_autotuner_picks_a_schedule_and_keeps_results():
    spec = _case("mixture")
    with Engine(spec) as eng:
        eng.run(10)
        t = eng.tuning()
        assert t["autotuned"] and t["threads_per_particle"] in (1, 2, 4)
        auto = eng.state()
    with Engine(spec) as eng:
        eng.set_tuning(1, True, 8, False)
        eng.run(10)
        fixed = eng.state()
    for key in ("positions", "velocities", "forces"):
        assert np.array_equal(auto[key], fixed[key]), key


def test_invalid_schedule_is_rejected():
    with Engine(_case("mixture")) as eng:
        with pytest.raises(ValueError):
            eng.set_tuning(3, True)
        with pytest.raises(ValueError):
            eng.set_tuning(2, True, 6)
