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

Beside each module it links ``_ref_neighbors`` from ``oracle/ref_neighbors.cu``
(a checker of this repository) with the same reference objects, minus the
reference's PYBIND11_MODULE translation unit: ``neighbor_dump(spec)`` returns
the list the reference's own NeighborSystem builds for a spec.

    python oracle/build_ref.py [<reference checkout>] [--jobs 8]

Without an argument the checkout is $BEADS_REFERENCE_SRC, else the path this
recipe was written against (/root/reference); when neither exists the recipe
prints why and builds nothing.
"""

from __future__ import annotations

import argparse
import concurrent.futures
import os
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
    build_harness(ref, precision, objdir, [o for o in objs if o.name != "bindings__module.cpp.o"])
    return target


def build_harness(ref: pathlib.Path, precision: str, objdir: pathlib.Path,
                  objs: list[pathlib.Path]) -> pathlib.Path:
    """Links oracle/ref_neighbors.cu against the reference's objects."""
    defines = ["-DBEADS_REAL64"] if precision == "f64" else []
    src = HERE / "ref_neighbors.cu"
    obj = objdir / "harness__ref_neighbors.cu.o"
    suffix = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    target = OUT / precision / f"_ref_neighbors{suffix}"
    if not (obj.exists() and obj.stat().st_mtime >= src.stat().st_mtime):
        cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
               "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", *defines, *includes(ref),
               "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"{src}:\n{r.stderr[-4000:]}")
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler",
           "-fPIC", str(obj), *map(str, objs), "-lpthread", "-o", str(target)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-4000:])
    return target


def default_reference() -> pathlib.Path:
    return pathlib.Path(os.environ.get("BEADS_REFERENCE_SRC", "/root/reference"))


def built() -> bool:
    """True when both precisions' _native and _ref_neighbors modules exist."""
    return all(list((OUT / p).glob(f"{m}*.so")) for p in ("f32", "f64")
               for m in ("_native", "_ref_neighbors"))


def main() -> None:
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("reference", type=pathlib.Path, nargs="?", default=None)
    parser.add_argument("--jobs", type=int, default=8)
    parser.add_argument("--precision", choices=["f32", "f64", "both"], default="both")
    args = parser.parse_args()
    if args.reference is None:
        args.reference = default_reference()
        if not (args.reference / "native" / "src").is_dir():
            print(f"reference checkout not found at {args.reference}; checker modules not built")
            return
    for p in (["f32", "f64"] if args.precision == "both" else [args.precision]):
        print(build(args.reference.resolve(), p, args.jobs))
    sys.stdout.flush()


if __name__ == "__main__":
    main()
