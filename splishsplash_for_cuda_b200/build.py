"""Builds the sm_100a shared library of the DFSPH time step (libdfsph_b200.so) in-tree.

Usage: python -m splishsplash_for_cuda_b200.build [--force]

Each CUDA translation unit is compiled with nvcc for sm_100a only (host-only C++ files with g++),
then linked into one shared library with the static CUDA runtime and zlib (for .bgeo files). The library has a plain C ABI (include/dfsph_c.h) and no
dependency on PyTorch.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "libdfsph_b200.so"
OBJ = PKG / "_build"
# The checked variant: every cell-table run, neighbour-list entry and list count is range-checked on
# the device after each neighbour search (DFSPH_ST_INDEX instead of an out-of-range read); the solver
# passes are the product's code. For debugging and the tests.
CHECKED_OUT = PKG / "libdfsph_b200_checked.so"
CHECKED_OBJ = PKG / "_build_checked"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC,-O3",
    "-I",
    str(ROOT / "include"),
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libdfsph_b200.so")


CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-I", str(ROOT / "include")]


def cxx() -> str:
    for cand in (os.environ.get("CXX"), shutil.which("g++"), "/usr/bin/g++"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("g++ not found")


def sources() -> list[Path]:
    """CUDA translation units (nvcc) and host-only C++ files (g++)."""
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra_flags: list[str] | None = None,
          out: Path | None = None, obj_dir: Path | None = None) -> Path:
    """Compiles every csrc/*.cu for sm_100a and links libdfsph_b200.so (or `out`). Returns its path."""
    OUT_ = Path(out) if out is not None else OUT
    OBJ_ = Path(obj_dir) if obj_dir is not None else OBJ
    OBJ_.mkdir(parents=True, exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((ROOT / "include").glob("*.h"))
    flags = NVCC_FLAGS + (extra_flags or [])
    jobs = []
    objs = []
    for src in sources():
        obj = OBJ_ / (src.stem + src.suffix.replace(".", "_") + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            if src.suffix == ".cpp":
                jobs.append([cxx(), *CXX_FLAGS, "-c", str(src), "-o", str(obj)])
            else:
                jobs.append([nvcc(), *flags, "-c", str(src), "-o", str(obj)])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            results = list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), jobs))
        for cmd, res in zip(jobs, results):
            if verbose or res.returncode != 0:
                sys.stderr.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
            if res.returncode != 0:
                raise RuntimeError(f"compile failed for {cmd[-3]}")
    if force or jobs or _stale(OUT_, objs):
        link = [nvcc(), *ARCH, "-shared", "-o", str(OUT_), *map(str, objs), "-cudart", "static", "-lz"]
        res = subprocess.run(link, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(" ".join(link) + "\n" + res.stdout + res.stderr)
            raise RuntimeError("link of libdfsph_b200.so failed")
    return OUT_


def build_checked(force: bool = False, verbose: bool = False) -> Path:
    """Builds libdfsph_b200_checked.so (-DDFSPH_CHECKED) beside the product library."""
    return build(force=force, verbose=verbose, extra_flags=["-DDFSPH_CHECKED"], out=CHECKED_OUT,
                 obj_dir=CHECKED_OBJ)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers/spills per kernel")
    ap.add_argument("--checked", action="store_true", help="also build libdfsph_b200_checked.so")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_info else None
    print(build(force=a.force or a.ptxas_info, verbose=a.verbose or a.ptxas_info, extra_flags=extra))
    if a.checked:
        print(build_checked(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    main()
