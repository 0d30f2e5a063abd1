"""The CPU oracle's neighbour sets against the reference engine's OWN lists.

tests/golden/ref_nbr_<case>.npz hold the list the reference's engine built
for each input (its NeighborSystem driven by oracle/ref_neighbors.cu and
linked with its own objects; tests/golden/make_reference_neighbor_fixtures.py),
by tag: list lengths, an order-free hash of every row's partner tags, the
sorted partner rows for the small cases, the hash over all rows, the build
path and the excluded-pair count.  Cases: the three committed reference
specs (LJ lattice, binary mixture, bead-spring chains with 1-2/1-3
exclusions) and seeded generated inputs that cover every build path and the
benchmark sizes: the 1,048,576-bead mixture in its 37.2 nm box, a 65,536-bead
mixture, a 20,000-bead melt with exclusions, a small-dimension grid
(5 x 5 x 2 cells), a direct grid (2 x 2 x 2) and crowded cells (~64 per cell).

Bar: the sets are equal, row by row, skin shell included.
"""

from __future__ import annotations

import numpy as np
import pytest

from beads_b200.engine import ReplicaSpec
from oracle import oracle as O
from tests.conftest import ROOT
from tests.golden.make_reference_neighbor_fixtures import (COMMITTED, GENERATED, generated_case,
                                                            input_digest)
from tests.helpers import oracle_neighbors, partner_hash, partner_hash_all
from tests.test_reference_pin import fixture, tag_ordered

GOLDEN = ROOT / "tests" / "golden"
CASES = [*COMMITTED, *GENERATED]


def reference_lists(name: str):
    return np.load(GOLDEN / f"ref_nbr_{name}.npz")


def case_input(name: str) -> ReplicaSpec:
    """The input of case `name` with rows in tag order (row t - 1 is tag t)."""
    if name in COMMITTED:
        return tag_ordered(fixture(name)[1])
    return generated_case(name)


def assert_lists_match(ref, counts, partners_tags, name: str) -> None:
    """counts[n] and 1-based partner tags [n, cap] in tag order against the
    reference's fixture."""
    counts = np.asarray(counts)
    assert counts.shape == ref["counts"].shape, name
    bad = np.nonzero(counts != ref["counts"])[0]
    assert bad.size == 0, (name, "list lengths differ at rows", bad[:10].tolist())
    hashes = partner_hash(counts, partners_tags)
    if "rows" in ref.files:
        rows = ref["rows"]
        bad = np.nonzero(hashes[rows] != ref["hashes"])[0]
    else:
        bad = np.nonzero(hashes != ref["hashes"])[0]
    assert bad.size == 0, (name, "partner sets differ at rows", bad[:10].tolist())
    assert partner_hash_all(hashes) == int(ref["hash_all"]), name
    if "partners" in ref.files:
        want = ref["partners"]
        cap = want.shape[1]
        got = np.full((counts.shape[0], cap), 0xFFFFFFFF, np.uint32)
        width = min(cap, partners_tags.shape[1])
        live = np.arange(width)[None, :] < counts[:, None]
        got[:, :width] = np.where(live, partners_tags[:, :width], np.uint32(0xFFFFFFFF))
        assert np.array_equal(np.sort(got, axis=1), want), name


def test_fixtures_cover_every_path():
    paths = {str(reference_lists(name)["path"]) for name in CASES}
    assert paths == {"direct", "regular_cell", "small_dimension"}
    assert all(int(reference_lists(name)["overflow"]) == 0 for name in CASES)


@pytest.mark.parametrize("name", GENERATED)
def test_generated_inputs_are_the_fixture_inputs(name):
    assert input_digest(generated_case(name)) == str(reference_lists(name)["input_digest"])


@pytest.mark.parametrize("name", CASES)
def test_oracle_neighbor_sets_equal_the_reference_lists(name):
    ref = reference_lists(name)
    spec = case_input(name)
    cap = max(int(spec.max_neighbors), int(ref["counts"].max()))
    counts, partners = oracle_neighbors(spec, cap=cap)
    assert_lists_match(ref, counts, partners + 1, name)
    assert O.plan(spec.box_bound, spec.cutoff, spec.cutoff_buffer)["path"] == str(ref["path"])
    if spec.exclusion_distance and spec.bonds is not None:
        n_excl = O.exclusion_pairs(spec.n, spec.bonds, spec.exclusion_distance).shape[0]
        assert n_excl == int(ref["excluded_pairs"])
