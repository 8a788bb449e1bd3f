"""Build the CUDA library libsmoke_b200.so in-tree for sm_100a.

    python python-game-engine_b200/build.py        (or __graft_entry__.build())

Each csrc/*.cu is compiled to an object with nvcc (-gencode arch=compute_100a,code=sm_100a),
then linked into lib/libsmoke_b200.so against the shared CUDA runtime. The operator unit
is compiled with -fmad=false so that its float32/float64 arithmetic rounds exactly as the
reference's Numba kernels do; the solver units keep FMA contraction.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(HERE, "lib")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(LIBDIR, "libsmoke_b200.so")
LIB_BC = os.path.join(LIBDIR, "libsmoke_b200_bc.so")
OBJDIR_BC = os.path.join(HERE, "_build_bc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC]
PER_FILE = {"operators.cu": ["-fmad=false"], "batch.cu": ["-fmad=false"], "rbsor_split.cu": ["-fmad=false"]}


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _build_one(nvcc, lib, objdir, extra, verbose, force):
    os.makedirs(objdir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(INCLUDE, "smoke_b200.h"))
    objs = []
    for src in sources():
        s = os.path.join(CSRC, src)
        o = os.path.join(objdir, src[:-3] + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers + [__file__]):
            cmd = [nvcc, *ARCH, *COMMON, *PER_FILE.get(src, []), *extra, "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _stale(lib, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", lib, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return lib


def build(verbose: bool = False, force: bool = False, bounds_check: bool = True) -> str:
    """Build lib/libsmoke_b200.so and, with bounds_check, lib/libsmoke_b200_bc.so (the same
    sources with -DSG_BOUNDS_CHECK=1: index checks in the tiled kernels, for tests)."""
    nvcc = _nvcc()
    os.makedirs(LIBDIR, exist_ok=True)
    if bounds_check:
        _build_one(nvcc, LIB_BC, OBJDIR_BC, ["-DSG_BOUNDS_CHECK=1"], verbose, force)
    return _build_one(nvcc, LIB, OBJDIR, [], verbose, force)


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv, bounds_check="--no-bounds-check" not in sys.argv))
