"""Build libbeads_b200.so in-tree with nvcc for sm_100a.

Usage: ``python -m beads_b200.build [--force]``.  Objects go to
``beads_b200/_build/``; the shared library to ``beads_b200/libbeads_b200.so``.
Each translation unit is rebuilt when it or any header is newer than its
object.
"""

from __future__ import annotations

import argparse
import concurrent.futures
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libbeads_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-fvisibility=hidden",
    f"-I{ROOT / 'include'}",
]


def nvcc() -> str:
    found = shutil.which("nvcc")
    if found:
        return found
    candidate = "/usr/local/cuda/bin/nvcc"
    if os.path.exists(candidate):
        return candidate
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build beads_b200")


def sources() -> list[pathlib.Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def headers() -> list[pathlib.Path]:
    return sorted(list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + list((ROOT / "include").glob("*.h")))


def _compile(src: pathlib.Path, force: bool, extra: list[str]) -> pathlib.Path:
    obj = BUILD / (src.name + ".o")
    newest_header = max((h.stat().st_mtime for h in headers()), default=0.0)
    if (
        not force
        and obj.exists()
        and obj.stat().st_mtime >= max(src.stat().st_mtime, newest_header)
    ):
        return obj
    cmd = [nvcc(), *ARCH, *COMMON, *extra, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cu":
        cmd[1:1] = ["-Xptxas", "-v"] if os.environ.get("BEADS_PTXAS_VERBOSE") else []
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{result.stdout}\n{result.stderr}")
    if result.stderr.strip() and os.environ.get("BEADS_PTXAS_VERBOSE"):
        sys.stderr.write(result.stderr)
    return obj


def build(force: bool = False, jobs: int | None = None) -> pathlib.Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sources()
    extra: list[str] = []
    with concurrent.futures.ThreadPoolExecutor(max_workers=jobs or min(8, len(srcs))) as pool:
        objs = list(pool.map(lambda s: _compile(s, force, extra), srcs))
    if (
        not force
        and LIB.exists()
        and LIB.stat().st_mtime >= max(o.stat().st_mtime for o in objs)
    ):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", *map(str, objs), "-o", str(tmp)]
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"link failed:\n{result.stdout}\n{result.stderr}")
    os.replace(tmp, LIB)
    return LIB


def main() -> None:
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("--force", action="store_true")
    args = parser.parse_args()
    print(build(force=args.force))


if __name__ == "__main__":
    main()
