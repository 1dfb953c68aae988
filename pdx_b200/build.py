"""Builds libpdx_b200.so (the C-ABI engine) in-tree with nvcc for sm_100a.

Each .cu file compiles to its own object in parallel (pdx_b200/_build/), then one link step
makes the shared library; no device code is called across files, so no relocatable device code
is needed.

Usage: python -m pdx_b200.build [--verbose] [--ptxas]
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpdx_b200.so")
SOURCES = ["pdxg_index.cu", "pdxg_search.cu", "pdxg_toplevel.cu", "pdxg_start.cu", "pdxg_probe.cu",
           "pdxg_rotate.cu", "pdxg_noalloc.cu", "pdxg_gemm.cu", "pdxg_build.cu", "pdxg_maint.cu",
           "pdxg_scan.cu"]
HEADERS = ["pdxg_common.cuh", "pdxg_block.cuh", "pdxg_gemm.cuh", "pdxg_engine.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-ccbin", "/usr/bin/g++"]


def _deps():
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "pdx_b200.h"))
    return deps


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in _deps() if os.path.exists(p))


def _obj(src: str) -> str:
    return os.path.join(OBJ, os.path.splitext(src)[0] + ".o")


def _obj_stale(src: str) -> bool:
    o = _obj(src)
    if not os.path.exists(o):
        return True
    t = os.path.getmtime(o)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", "pdx_b200.h")]
    return any(os.path.getmtime(p) > t for p in [os.path.join(CSRC, src)] + hdrs if os.path.exists(p))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout, r.stderr, flush=True)


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    todo = [s for s in SOURCES if force or extra or _obj_stale(s)]
    cmds = [[NVCC, *ARCH, *FLAGS, *(extra or []), "-c", "-o", _obj(s), os.path.join(CSRC, s)] for s in todo]
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_run, c, verbose) for c in cmds]:
            f.result()
    _run([NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-ccbin", "/usr/bin/g++", "-o", LIB,
          *[_obj(s) for s in SOURCES], "-lcudart"], verbose)
    return LIB


if __name__ == "__main__":
    v = "--verbose" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else None
    print(build(force=True, verbose=v or extra is not None, extra=extra))
