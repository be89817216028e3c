"""Builds libemerge_cuda.so in-tree for sm_100a.

    python -m emerge_engine_b200.build [--force]

Physics translation units are compiled with -fmad=false (no a*b+c contraction, matching
the Rust reference, which never contracts) and IEEE division / square root.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(PKG, "libemerge_cuda.so")
SOURCES = ["step_kernels.cu", "det_kernels.cu", "sort.cu", "sort_noalloc.cu", "sim.cu"]
HEADERS = ["physics.cuh", "device_state.cuh", "kernels.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "nvcc")


def _stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(PKG, "..", "include", "emerge_cuda.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return OUT
    cmd = [NVCC, *ARCH, "-O3", "-std=c++17", "-lineinfo", "-fmad=false",
           "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared", "-o", OUT]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, f) for f in SOURCES]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
