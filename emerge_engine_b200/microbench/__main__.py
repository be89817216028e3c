"""Builds and runs the floor microbenchmarks (microbench/floor.cu) on cuda:0 and prints
their JSON line: the per-launch times of the particle passes' memory components alone
(scatter reductions, stencil gather, state streaming) for 1M particles at 4 per cell."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "floor")


def build() -> str:
    src = os.path.join(HERE, "floor.cu")
    if not os.path.exists(BIN) or os.path.getmtime(BIN) < os.path.getmtime(src):
        subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                        "-lineinfo", "-o", BIN, src], check=True)
    return BIN


if __name__ == "__main__":
    sys.exit(subprocess.run([build()] + sys.argv[1:]).returncode)
