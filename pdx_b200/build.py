"""Builds libpdx_b200.so (the C-ABI engine) in-tree with nvcc for sm_100a.

Usage: python -m pdx_b200.build [--verbose]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libpdx_b200.so")
SOURCES = ["pdxg_index.cu", "pdxg_search.cu", "pdxg_toplevel.cu", "pdxg_start.cu", "pdxg_probe.cu",
           "pdxg_rotate.cu", "pdxg_noalloc.cu", "pdxg_gemm.cu", "pdxg_build.cu", "pdxg_maint.cu"]
HEADERS = ["pdxg_common.cuh", "pdxg_block.cuh", "pdxg_gemm.cuh", "pdxg_engine.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-shared",
         "--expt-relaxed-constexpr", "-ccbin", "/usr/bin/g++"]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "pdx_b200.h"))
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    if not force and not _stale():
        return LIB
    cmd = [NVCC, *ARCH, *FLAGS, *(extra or []), "-o", LIB,
           *[os.path.join(CSRC, s) for s in SOURCES], "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout, r.stderr)
    return LIB


if __name__ == "__main__":
    v = "--verbose" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else None
    print(build(force=True, verbose=v or extra is not None, extra=extra))
