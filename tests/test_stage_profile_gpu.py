"""The stage profiler times each stage of a small lattice step."""

from __future__ import annotations

import pytest

from tests import stage_profile

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("stage", ["forces", "forces_kick", "rebuild", "step"])
def test_stage_profile_reports_positive_time(stage):
    out = stage_profile.main(["--workload", "lattice", "--beads", "4096", "--stage", stage,
                              "--reps", "3", "--warm", "5"])
    assert out["stage"] == stage and out["ms"] > 0.0
