"""Builds libemerge_cuda.so in-tree for sm_100a.

    python -m emerge_engine_b200.build [--force] [-v]

Each translation unit is compiled to an object under _build/ and the objects are linked
into one shared library.  Two arithmetic contracts:
  exact  -fmad=false (no a*b+c contraction, matching the Rust reference, which never
         contracts) with IEEE division and square root: the reference-order mode, the
         grid update, the controller, spawning and every host-visible reduction.
  fast   approximate (2-ulp) division and square root, except where the code asks for IEEE
         rounding (the SVD, polar decomposition and return mappings: physics.cuh esqrt /
         ediv), and no implicit contraction: the stencil sums of G2P and P2G use explicit
         fused multiply-adds; the constitutive arithmetic is left uncontracted, as in the
         reference.  Measured on the 160k-particle granular scene over 100 frames, implicit
         contraction moved region speeds by 1.5e-3 against the oracle, 14x what the
         reference itself moves when its particles are summed in another order; without it
         the fast path stays at that level (1.1e-4).  The fused pipeline's particle,
         density, contact and closure kernels use this contract.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(PKG, "libemerge_cuda.so")
BUILD_DIR = os.path.join(PKG, "_build")
EXACT = ["-fmad=false"]
FAST = ["-fmad=false", "-prec-div=false", "-prec-sqrt=false"]
SOURCES = {
    "step_kernels.cu": EXACT,
    "fast_kernels.cu": FAST,
    "det_kernels.cu": EXACT,
    "multifield.cu": EXACT,
    "multifield_fast.cu": FAST,
    "sort.cu": EXACT,
    "sort_noalloc.cu": EXACT,
    "sim.cu": EXACT,
    "closure.cu": FAST,
    "closure_tiles.cu": FAST,
    "batch.cu": EXACT,
    "nbody.cu": EXACT,
}
HEADERS = ["physics.cuh", "device_state.cuh", "kernels.h", "particle_pass.cuh", "closure.cuh", "closure_host.h",
           "multifield.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off"]
NVCC = os.environ.get("NVCC", "nvcc")


def _stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in list(SOURCES) + HEADERS]
    deps.append(os.path.join(PKG, "..", "include", "emerge_cuda.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src: str, flags: list[str], verbose: bool) -> str:
    obj = os.path.join(BUILD_DIR, os.path.splitext(src)[0] + ".o")
    cmd = [NVCC, *ARCH, *COMMON, *flags, "-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    subprocess.run(cmd, check=True)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return OUT
    os.makedirs(BUILD_DIR, exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda kv: _compile(kv[0], kv[1], verbose), SOURCES.items()))
    subprocess.run([NVCC, *ARCH, "-shared", "-o", OUT, *objs], check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
