"""Runs the reference engine's own extension module (built by
oracle/build_ref.py into oracle/_ref/) on a spec dict.

TEST INFRASTRUCTURE ONLY.  Both precisions export a module named ``_native``,
so each run happens in a fresh subprocess that loads exactly one of them.

    python -m oracle.ref <f32|f64> <spec.json> <spec.npz> <workdir>
    python -m oracle.ref <f32|f64> --many <root> <count>
    python -m oracle.ref <f32|f64> --neighbors <spec.json> <spec.npz> <out.npz>

runs ``_native.execute_simulation(spec)`` with ``workdir`` as the current
directory (the spec's output prefixes are relative to it); ``--many`` runs
<root>/0 .. <root>/<count-1> one after another in one process.
"""

from __future__ import annotations

import glob
import importlib.util
import json
import os
import pathlib
import subprocess
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent


def module_path(precision: str) -> pathlib.Path:
    found = glob.glob(str(HERE / "_ref" / precision / "_native*.so"))
    if not found:
        raise FileNotFoundError(f"reference module for {precision} is not built "
                                "(python oracle/build_ref.py <reference checkout>)")
    return pathlib.Path(found[0])


def available() -> bool:
    try:
        module_path("f32")
        module_path("f64")
        return True
    except FileNotFoundError:
        return False


def _load(precision: str):
    spec = importlib.util.spec_from_file_location("_native", module_path(precision))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def save_spec(spec: dict, json_path: pathlib.Path, npz_path: pathlib.Path) -> None:
    arrays: dict = {}

    def split(obj, path):
        if isinstance(obj, np.ndarray):
            arrays[path] = obj
            return {"__array__": path}
        if isinstance(obj, dict):
            return {k: split(v, f"{path}.{k}") for k, v in obj.items()}
        if isinstance(obj, (list, tuple)):
            return [split(v, f"{path}.{i}") for i, v in enumerate(obj)]
        return obj

    json_path.write_text(json.dumps(split(spec, "spec"), sort_keys=True))
    np.savez(npz_path, **arrays)


def load_spec(json_path: pathlib.Path, npz_path: pathlib.Path) -> dict:
    arrays = np.load(npz_path)

    def join(obj):
        if isinstance(obj, dict):
            if set(obj) == {"__array__"}:
                return arrays[obj["__array__"]]
            return {k: join(v) for k, v in obj.items()}
        if isinstance(obj, list):
            return [join(v) for v in obj]
        return obj

    return join(json.loads(json_path.read_text()))


def run(precision: str, spec: dict, workdir: pathlib.Path, timeout: float = 1800.0) -> None:
    """Runs the reference module of `precision` on `spec` in a subprocess."""
    workdir = pathlib.Path(workdir)
    workdir.mkdir(parents=True, exist_ok=True)
    jp, npz = workdir / "spec.json", workdir / "spec.npz"
    save_spec(spec, jp, npz)
    env = dict(os.environ)
    env["PYTHONPATH"] = str(ROOT) + os.pathsep + env.get("PYTHONPATH", "")
    subprocess.run([sys.executable, "-m", "oracle.ref", precision, str(jp), str(npz),
                    str(workdir)], check=True, env=env, timeout=timeout)


def harness_path(precision: str) -> pathlib.Path:
    found = glob.glob(str(HERE / "_ref" / precision / "_ref_neighbors*.so"))
    if not found:
        raise FileNotFoundError(f"reference neighbour harness for {precision} is not built "
                                "(python oracle/build_ref.py <reference checkout>)")
    return pathlib.Path(found[0])


def neighbors(precision: str, spec: dict, workdir: pathlib.Path,
              timeout: float = 1800.0) -> dict:
    """The reference engine's own neighbour list after its initial build for
    `spec` (oracle/ref_neighbors.cu), computed in a subprocess: counts[n] and
    partners[n][max_neighbors] in tag order, overflow, path, excluded_pairs."""
    workdir = pathlib.Path(workdir)
    workdir.mkdir(parents=True, exist_ok=True)
    jp, npz, out = workdir / "spec.json", workdir / "spec.npz", workdir / "neighbors.npz"
    save_spec(spec, jp, npz)
    env = dict(os.environ)
    env["PYTHONPATH"] = str(ROOT) + os.pathsep + env.get("PYTHONPATH", "")
    subprocess.run([sys.executable, "-m", "oracle.ref", precision, "--neighbors", str(jp),
                    str(npz), str(out)], check=True, env=env, timeout=timeout)
    with np.load(out) as data:
        return {k: data[k] for k in data.files}


def run_many(precision: str, specs: list[dict], workdir: pathlib.Path,
             timeout: float = 3600.0) -> list[pathlib.Path]:
    """Runs every spec in turn in ONE subprocess (one module load); spec k runs
    in workdir/k.  Returns the run directories."""
    workdir = pathlib.Path(workdir)
    dirs = []
    for k, spec in enumerate(specs):
        d = workdir / str(k)
        d.mkdir(parents=True, exist_ok=True)
        save_spec(spec, d / "spec.json", d / "spec.npz")
        dirs.append(d)
    env = dict(os.environ)
    env["PYTHONPATH"] = str(ROOT) + os.pathsep + env.get("PYTHONPATH", "")
    subprocess.run([sys.executable, "-m", "oracle.ref", precision, "--many", str(workdir),
                    str(len(specs))], check=True, env=env, timeout=timeout)
    return dirs


def _prepare(spec: dict, precision: str) -> dict:
    if precision == "f64":
        # The double build takes float64 reals; the float32 inputs convert exactly.
        for key in ("box_bound", "positions", "velocities", "masses"):
            spec["system"][key] = np.ascontiguousarray(spec["system"][key], dtype=np.float64)
    return spec


def main(argv: list[str]) -> None:
    if len(argv) == 5 and argv[1] == "--neighbors":
        precision, _, jp, npz, out = argv
        spec = _prepare(load_spec(pathlib.Path(jp), pathlib.Path(npz)), precision)
        hs = importlib.util.spec_from_file_location("_ref_neighbors", harness_path(precision))
        mod = importlib.util.module_from_spec(hs)
        hs.loader.exec_module(mod)
        d = mod.neighbor_dump(spec)
        np.savez(out, counts=d["counts"], partners=d["partners"], overflow=d["overflow"],
                 path=np.array(d["path"]), excluded_pairs=d["excluded_pairs"],
                 builds=d["builds"])
        return
    if len(argv) == 4 and argv[1] == "--many":
        precision, _, root, count = argv
        mod = _load(precision)
        for k in range(int(count)):
            d = pathlib.Path(root) / str(k)
            spec = _prepare(load_spec(d / "spec.json", d / "spec.npz"), precision)
            os.chdir(d)
            mod.execute_simulation(spec)
        return
    precision, jp, npz, workdir = argv
    spec = _prepare(load_spec(pathlib.Path(jp), pathlib.Path(npz)), precision)
    mod = _load(precision)
    os.chdir(workdir)
    mod.execute_simulation(spec)


if __name__ == "__main__":
    main(sys.argv[1:])
