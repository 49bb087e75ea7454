"""Build the CUDA library in-tree with nvcc for sm_100a.

``python -m chiaro_b200.build`` compiles ``csrc/stage.cu`` (which includes
every kernel header) into ``chiaro_b200/_build/libchiaro_depth.so``, and the
host-only check library ``libchiaro_hostcheck.so`` that lets CPU tests run
the device math restatements on the host.

Flags: ``-fmad=false`` keeps every multiply and add separately rounded, as the
reference computes them; division and square root stay IEEE (the defaults).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT = PKG / "_build"
LIB = OUT / "libchiaro_depth.so"
HOSTCHECK = OUT / "libchiaro_hostcheck.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-O2,-ffp-contract=off",
              "--expt-relaxed-constexpr", "-Xptxas", "-O3"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA library cannot be built")


def _sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.inc")) + \
        sorted(CSRC.glob("*.cpp")) + [INCLUDE / "chiaro_depth.h"]


def _stale(target: Path) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in _sources())


def build(force: bool = False, verbose: bool = False) -> Path:
    OUT.mkdir(exist_ok=True)
    if force or _stale(LIB):
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-shared", "-o", str(LIB), str(CSRC / "stage.cu"),
               "-cudart", "static"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True, cwd=str(CSRC))
    if force or _stale(HOSTCHECK):
        cxx = os.environ.get("CXX", "g++")
        cuda_inc = Path(nvcc()).resolve().parent.parent / "include"
        cmd = [cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
               f"-I{cuda_inc}", "-o", str(HOSTCHECK), str(CSRC / "hostcheck.cpp")]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True, cwd=str(CSRC))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
