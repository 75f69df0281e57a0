"""Builds libaxr.so (the sm_100a kernels and the C ABI) in-tree.

    python -m axi_visualizer_b200.build [--verbose]

nvcc cross-compiles for sm_100a without a GPU.  -fmad=false keeps every
multiply and add separately rounded, which the bit-exact coverage, triangle
ids and depth rely on (division and square root stay IEEE by default).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libaxr.so")
SOURCES = [os.path.join(CSRC, "axr.cu")]
DEPS = SOURCES + [os.path.join(CSRC, f) for f in ("raster.cuh", "kernels.cuh", "batch.cuh", "shadow_tiles.cuh")] + [
    os.path.join(HERE, "..", "include", "axr.h")]

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
         "-prec-div=true", "-prec-sqrt=true", "-Xcompiler", "-fPIC", "-shared", "-lcudart"]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in DEPS)


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    if not force and not needs_build():
        return LIB
    cmd = [NVCC, *FLAGS, *extra, "-o", LIB, *SOURCES]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    v = "--verbose" in sys.argv or "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(force=True, verbose=v, extra=extra))
