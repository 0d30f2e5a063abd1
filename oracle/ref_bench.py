"""Times the reference engine's own float32 build and beads_b200 on the same
spec dicts, through each engine's ``execute_simulation``, using the
reference's own timer (the ``steps_per_second`` line of its log,
native/src/simulation/output/log/log_output.cpp:370-404, which covers the
initial neighbour build and every step).

TEST INFRASTRUCTURE ONLY (needs a GPU and oracle/build_ref.py's output).

    python -m oracle.ref_bench <out.json> [--quick] [--replicas | --chains]
"""

from __future__ import annotations

import json
import pathlib
import re
import sys
import tempfile

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests" / "golden"))

from beads_b200 import _native, workloads  # noqa: E402
from beads_b200.engine import Engine  # noqa: E402
from make_reference_fixtures import spec_for  # noqa: E402
from oracle import ref  # noqa: E402


def _sps(log_path: pathlib.Path) -> float:
    m = re.search(r"steps_per_second\s+: ([0-9.eE+-]+)", log_path.read_text())
    return float(m.group(1))


def _relaxed_mixture(n: int):
    box = 37.2 * (n / 1_048_576) ** (1 / 3)
    spec = workloads.lj_mixture(n=n, box=box, seed=3)
    cap = spec.max_neighbors
    spec.max_neighbors = 256
    with Engine(spec) as eng:
        eng.minimize(500, 0.004, 200.0)
        spec.positions = workloads._inside(eng.state()["positions"].astype(np.float64),
                                           np.zeros(3), np.full(3, box))
    spec.max_neighbors = cap
    return spec


def reference_engine_rate(r, steps: int) -> dict:
    """The reference engine's own float32 build on replica `r` through its
    execute_simulation (a thermo row at the end only), timed by its own log
    (steps_per_second: wall time of the whole run, initial build included).
    Returns the steps, its steps/s and atom-steps/s."""
    spec = spec_for(r, steps, "run", forces=False, thermo_every=steps)
    with tempfile.TemporaryDirectory() as tmp:
        tmp = pathlib.Path(tmp)
        ref.run("f32", spec, tmp / "ref")
        sps = _sps(tmp / "ref" / "run.log")
    return {"steps": steps, "steps_per_second": sps, "atom_steps_per_s": sps * r.n}


def _replica_batch(steps: int, count: int) -> dict:
    """The uneven 512-replica batch: the reference engine one replica at a
    time (its own timer per run, summed) against one batched beads_b200 engine
    (wall time of the whole run(), including its first neighbour build and
    schedule autotuning)."""
    import time

    specs = workloads.replica_batch(count)
    atoms = sum(r.n for r in specs)
    with tempfile.TemporaryDirectory() as tmp:
        dirs = ref.run_many("f32", [spec_for(r, steps, "run", forces=False, thermo_every=steps)
                                    for r in specs], pathlib.Path(tmp))
        ref_s = sum(steps / _sps(d / "run.log") for d in dirs)
    with Engine(specs) as eng:
        eng.eval()
        t0 = time.perf_counter()
        eng.run(steps)
        ours_s = time.perf_counter() - t0
    return {"replicas": count, "atoms": atoms, "steps": steps,
            "reference_sequential_s": ref_s,
            "reference_atom_steps_per_s": atoms * steps / ref_s,
            "ours_batched_s": ours_s, "ours_atom_steps_per_s": atoms * steps / ours_s,
            "speedup": ref_s / ours_s}


def main(argv: list[str]) -> None:
    out_path = pathlib.Path(argv[0])
    quick = "--quick" in argv
    if "--replicas" in argv:
        entry = _replica_batch(100 if quick else 500, 64 if quick else 512)
        print("replicas", json.dumps(entry))
        out_path.write_text(json.dumps({"replica_batch": entry}, indent=1))
        return
    # Step counts of the workloads' own specifications: the 4096-bead lattice
    # runs 1,000 steps, the 1M-bead mixture 10,000, the 400,000-bead melt 20,000.
    if "--chains" in argv:
        n_chains = 250 if quick else 2000
        melt = workloads.relaxed(workloads.polymer_melt(n_chains=n_chains, growth="lockstep"))
        cases = [(f"chains_{melt.n}", melt, 1000 if quick else 20000)]
    else:
        cases = [("lattice_4096", workloads.lj_lattice(n_side=16), 1000)]
        n_mix = 131072 if quick else 1_048_576
        cases.append((f"mixture_{n_mix}", _relaxed_mixture(n_mix), 200 if quick else 10000))
    results = {}
    for name, r, steps in cases:
        spec = spec_for(r, steps, "run", forces=False, thermo_every=steps)
        entry = {"n": r.n, "steps": steps}
        with tempfile.TemporaryDirectory() as tmp:
            tmp = pathlib.Path(tmp)
            ref.run("f32", spec, tmp / "ref")
            entry["reference_steps_per_second"] = _sps(tmp / "ref" / "run.log")
            (tmp / "ours").mkdir()
            import os

            cwd = os.getcwd()
            os.chdir(tmp / "ours")
            try:
                _native.execute_simulation(spec)
            finally:
                os.chdir(cwd)
            entry["ours_steps_per_second"] = _sps(tmp / "ours" / "run.log")
        entry["reference_atom_steps_per_s"] = entry["reference_steps_per_second"] * r.n
        entry["ours_atom_steps_per_s"] = entry["ours_steps_per_second"] * r.n
        entry["speedup"] = entry["ours_steps_per_second"] / entry["reference_steps_per_second"]
        results[name] = entry
        print(name, json.dumps(entry))
    out_path.write_text(json.dumps(results, indent=1))


if __name__ == "__main__":
    main(sys.argv[1:])
