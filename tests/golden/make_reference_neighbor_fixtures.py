"""Generates tests/golden/ref_nbr_<case>.npz: the reference engine's OWN
neighbour list after its initial build, by tag.

Needs a GPU and the reference's checker modules built by
``python oracle/build_ref.py <reference checkout>`` (``_ref_neighbors``:
oracle/ref_neighbors.cu linked with the reference's objects).  For every case
the same spec dict goes to the reference (float32 build, the precision the
list decisions are pinned in) and, in the tests, to the oracle and to the CUDA
engine.

Inputs: the three committed reference specs (tests/golden/ref_<case>_spec.*)
and seeded generated systems that cover every build path and the sizes the
benchmarks run at (the 1,048,576-bead mixture at its 37.2 nm box, a melt with
1-2/1-3 exclusions, a small-dimension grid, a direct grid, crowded cells).
Generated inputs are rebuilt by the tests from the same seeds; each fixture
keeps a digest of its input arrays so a drifting generator fails loudly.

What is stored, per tag row (1-based tag t at row t - 1): the list length as
the reference stores it (``counts``) and an order-free 64-bit hash of the
partner tags (``hashes``, tests.helpers.partner_hash); the small cases also
keep the sorted partner lists themselves.  For the 1M-bead case the per-row
hashes are kept for a seeded sample of rows only, plus the hash over all rows
(``hash_all``), to keep the fixture small.

    python tests/golden/make_reference_neighbor_fixtures.py <output dir> [case ...]
"""

from __future__ import annotations

import hashlib
import pathlib
import sys
import tempfile

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from beads_b200 import workloads  # noqa: E402
from beads_b200.engine import ReplicaSpec  # noqa: E402
from tests.helpers import partner_hash, partner_hash_all  # noqa: E402

GOLDEN = ROOT / "tests" / "golden"
COMMITTED = ("lattice", "mixture", "chains")
GENERATED = ("mixture_1m", "mixture_64k", "melt_20k", "small_dim", "direct", "crowded")
FULL_LISTS_UP_TO = 5000      # cases up to this size also keep the partner lists
SAMPLE_ROWS = 20000          # per-row hashes kept for the 1M-bead case


def _uniform(n: int, box, seed: int, *, sigma, epsilon, cutoff: float, skin: float,
             max_neighbors: int, units: str = "reduced", types: int = 1) -> ReplicaSpec:
    """n beads uniform in an orthorhombic box (edges `box`), seeded."""
    rng = np.random.default_rng(seed)
    box = np.asarray(box, np.float64)
    lo = np.zeros(3)
    pos = workloads._inside(rng.uniform(0.0, 1.0, size=(n, 3)) * box, lo, box)
    t = np.ones(n, np.int32)
    if types == 2:
        t[rng.permutation(n)[: n // 5]] = 2
    masses = np.ones(n)
    vel = workloads._gaussian_velocities(np.random.default_rng(seed + 1), n, masses, 1.0)
    return ReplicaSpec(
        positions=pos, types=t, box_bound=np.array([lo, box], np.float32),
        epsilon=np.asarray(epsilon, np.float64), sigma=np.asarray(sigma, np.float64),
        cutoff=cutoff, dt=0.005, units=units, velocities=vel, masses=masses.astype(np.float32),
        shift=True, cutoff_buffer=skin, max_neighbors=max_neighbors, sort_every_rebuild=1)


def generated_case(name: str) -> ReplicaSpec:
    """The seeded input of a generated case (rebuilt identically by the tests)."""
    if name == "mixture_1m":
        # The benchmark mixture's composition, density and 37.2 nm box, from its
        # uniform start (the list rule does not depend on relaxation); a larger
        # capacity than the benchmark's 128 holds the unrelaxed fluctuations.
        return workloads.lj_mixture(n=1_048_576, box=37.2, seed=3, max_neighbors=192)
    if name == "mixture_64k":
        return workloads.lj_mixture(n=65536, box=(65536 / 20.37) ** (1 / 3), seed=21,
                                    max_neighbors=192)
    if name == "melt_20k":
        return workloads.polymer_melt(n_chains=100, beads=200, seed=23, growth="lockstep")
    if name == "small_dim":
        # 5 x 5 x 2 cells: the small-dimension path.
        return _uniform(1100, (14.0, 14.0, 7.0), 29, sigma=[[1.0]], epsilon=[[1.0]],
                        cutoff=2.5, skin=0.3, max_neighbors=160)
    if name == "direct":
        # 2 x 2 x 2 cells: the direct path.
        return _uniform(300, (7.0, 7.0, 7.0), 31, sigma=[[1.0]], epsilon=[[1.0]],
                        cutoff=2.5, skin=0.3, max_neighbors=320)
    if name == "crowded":
        # 4 x 4 x 4 cells of ~64 beads.
        return _uniform(4096, (3.2, 3.2, 3.2), 37, sigma=workloads.MIXTURE_SIG,
                        epsilon=workloads.MIXTURE_EPS, cutoff=0.6, skin=0.1,
                        max_neighbors=320, units="nm_kjmol", types=2)
    raise KeyError(name)


def input_digest(r: ReplicaSpec) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(r.positions, np.float32).tobytes())
    h.update(np.ascontiguousarray(r.types, np.int32).tobytes())
    h.update(np.ascontiguousarray(r.box_bound, np.float32).tobytes())
    if r.bonds is not None:
        h.update(np.ascontiguousarray(r.bonds, np.uint32).tobytes())
    return h.hexdigest()


def sample_rows(n: int) -> np.ndarray:
    return np.sort(np.random.default_rng(12345).choice(n, size=min(n, SAMPLE_ROWS),
                                                       replace=False))


def native_spec(name: str) -> dict:
    """The spec dict both engines receive for case `name`."""
    from oracle import ref

    if name in COMMITTED:
        return ref.load_spec(GOLDEN / f"ref_{name}_spec.json", GOLDEN / f"ref_{name}_spec.npz")
    from tests.golden.make_reference_fixtures import spec_for

    return spec_for(generated_case(name), 0, "nb", forces=False, thermo_every=1)


def main(out_dir: str, only: list[str]) -> None:
    from oracle import ref

    out = pathlib.Path(out_dir)
    out.mkdir(parents=True, exist_ok=True)
    for name in (*COMMITTED, *GENERATED):
        if only and name not in only:
            continue
        spec = native_spec(name)
        with tempfile.TemporaryDirectory() as tmp:
            d = ref.neighbors("f32", spec, pathlib.Path(tmp))
        counts, partners = d["counts"], d["partners"]
        n = counts.shape[0]
        hashes = partner_hash(counts, partners)
        fx: dict = {"counts": counts.astype(np.uint32), "overflow": d["overflow"],
                    "path": d["path"], "excluded_pairs": d["excluded_pairs"],
                    "hash_all": np.array(partner_hash_all(hashes), np.uint64)}
        if name in GENERATED:
            fx["input_digest"] = np.array(input_digest(generated_case(name)))
        if n > 200_000:
            rows = sample_rows(n)
            fx["rows"] = rows.astype(np.uint32)
            fx["hashes"] = hashes[rows]
        else:
            fx["hashes"] = hashes
        if n <= FULL_LISTS_UP_TO:
            cap = int(counts.max()) if n else 0
            fx["partners"] = np.sort(np.where(np.arange(partners.shape[1])[None, :cap]
                                              < counts[:, None], partners[:, :cap],
                                              np.uint32(0xFFFFFFFF)), axis=1)
        np.savez_compressed(out / f"ref_nbr_{name}.npz", **fx)
        print("wrote", name, n, "path", str(d["path"]), "mean", float(counts.mean()),
              "max", int(counts.max()), "overflow", int(d["overflow"]), flush=True)


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2:])
