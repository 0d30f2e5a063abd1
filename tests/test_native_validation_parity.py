"""Spec dicts the builders accept but the engine must refuse: our
``_native.execute_simulation`` raises the exception type and message of the
reference's own compiled module (tests/golden/native_validation_expect.json,
from tests/golden/make_native_validation_fixtures.py).  The refusal comes
before any device work, so this runs without a GPU."""

from __future__ import annotations

import json

import pytest

import beads_b200
from beads_b200 import _native
from tests.conftest import ROOT
from tests.golden.make_native_validation_fixtures import CASES, build_spec, native_error

EXPECT = json.loads((ROOT / "tests" / "golden" / "native_validation_expect.json").read_text())


@pytest.mark.parametrize("name", sorted(EXPECT))
def test_native_refusal_matches_reference(name):
    assert native_error(_native.execute_simulation, build_spec(beads_b200, CASES[name])) == \
        EXPECT[name]
