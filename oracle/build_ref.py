"""Builds the reference engine's own extension module from its sources, for
use as a checker only (test fixtures and the reference timing).

TEST INFRASTRUCTURE ONLY: nothing in beads_b200 loads these modules.

The reference's CMake project is not used.  This recipe compiles the
reference's C++/CUDA sources where they lie (native/src/**, includes
native/include and native/src) plus its pybind11 bindings with nvcc for
sm_100a, in two precisions, and links

    oracle/_ref/f32/_native.cpython-*.so    (real_t = float, the default build)
    oracle/_ref/f64/_native.cpython-*.so    (real_t = double, BEADS_REAL64)

Each module exposes the reference's ``build_info()`` and
``execute_simulation(spec)``; load it with ``oracle.ref.load(precision)``.

    python oracle/build_ref.py <reference checkout> [--jobs 8]
"""

from __future__ import annotations

import argparse
import concurrent.futures
import pathlib
import subprocess
import sys
import sysconfig

HERE = pathlib.Path(__file__).resolve().parent
OUT = HERE / "_ref"


def sources(ref: pathlib.Path) -> list[pathlib.Path]:
    src = ref / "native" / "src"
    files = sorted(list(src.rglob("*.cu")) + list(src.rglob("*.cpp")))
    if not files:
        raise SystemExit(f"no sources under {src}")
    return files


def includes(ref: pathlib.Path) -> list[str]:
    import pybind11

    return [f"-I{ref / 'native' / 'include'}", f"-I{ref / 'native' / 'src'}",
            f"-I{pybind11.get_include()}", f"-I{sysconfig.get_paths()['include']}"]


def compile_one(src: pathlib.Path, ref: pathlib.Path, objdir: pathlib.Path, defines: list[str]):
    rel = src.relative_to(ref / "native" / "src")
    obj = objdir / (str(rel).replace("/", "__") + ".o")
    if obj.exists() and obj.stat().st_mtime >= src.stat().st_mtime:
        return obj
    lang = [] if src.suffix == ".cu" else ["-x", "cu"]
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
           "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", *defines, *includes(ref), *lang,
           "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{src}:\n{r.stderr[-4000:]}")
    return obj


def build(ref: pathlib.Path, precision: str, jobs: int) -> pathlib.Path:
    objdir = OUT / f"obj_{precision}"
    objdir.mkdir(parents=True, exist_ok=True)
    defines = ["-DBEADS_REAL64"] if precision == "f64" else []
    with concurrent.futures.ThreadPoolExecutor(max_workers=jobs) as pool:
        objs = list(pool.map(lambda s: compile_one(s, ref, objdir, defines), sources(ref)))
    suffix = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    target = OUT / precision / f"_native{suffix}"
    target.parent.mkdir(parents=True, exist_ok=True)
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler",
           "-fPIC", *map(str, objs), "-lpthread", "-o", str(target)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-4000:])
    return target


def main() -> None:
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("reference", type=pathlib.Path)
    parser.add_argument("--jobs", type=int, default=8)
    parser.add_argument("--precision", choices=["f32", "f64", "both"], default="both")
    args = parser.parse_args()
    for p in (["f32", "f64"] if args.precision == "both" else [args.precision]):
        print(build(args.reference.resolve(), p, args.jobs))
    sys.stdout.flush()


if __name__ == "__main__":
    main()
