"""Builder misuse raises what the reference's own package raises: the same
exception type and message, or nothing where the reference accepts the call
(tests/golden/validation_expect.json, from
tests/golden/make_validation_fixtures.py)."""

from __future__ import annotations

import json

import pytest

import beads_b200
from tests.conftest import ROOT
from tests.golden.make_validation_fixtures import CASES, run_case

EXPECT = json.loads((ROOT / "tests" / "golden" / "validation_expect.json").read_text())


@pytest.mark.parametrize("name", sorted(CASES))
def test_validation_matches_reference(name):
    assert run_case(beads_b200, CASES[name]) == EXPECT[name]
