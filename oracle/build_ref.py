"""Build oracle/_ref/libaxr_ref.so: the reference's own OpenCL C kernels for
the rasterizer hot path, compiled for the CPU.  TEST INFRASTRUCTURE ONLY.

The kernels are read where they lie in the reference checkout
(PyOpenCL27C/Pipe/*.c, PyOpenCL27C/Shaders/*.c), passed through a small
mechanical rewrite that maps OpenCL C syntax onto C++ (vector literals
`(float3)(a, b, c)` -> `make_float3(a, b, c)`, address-space qualifiers,
`__local` -> thread-local arrays the harness can preload), and piped into
g++ on stdin, so no copy of the reference source is written anywhere.  Only
object files and the shared library land in oracle/_ref/ (git-ignored).

The harness (oracle/ref_harness.cpp) restates the host orchestration of
PyOpenCL27C/Ops0.py (CLDraw.drawAll) and Ops.py (CLDraw.shadowMap) and runs
each kernel work-item by work-item.

Usage: python oracle/build_ref.py [--reference /path/to/AXI_Visualizer]
Exit status 0 with a message when the reference checkout is absent.
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT, "libaxr_ref.so")

# (namespace, path inside the reference checkout[, prelude]); a prelude is
# declared first inside the kernel's namespace
SAT_STORES = "typedef sat_u16 ushort;"
KERNELS = [
    ("ref_trisetup", "PyOpenCL27C/Pipe/trisetup.c"),
    ("ref_trisetup_cull", "PyOpenCL27C/Pipe/trisetup_cull.c"),
    ("ref_trisetup_ortho", "PyOpenCL27C/Pipe/trisetupOrtho.c"),
    ("ref_gather", "PyOpenCL27C/Pipe/gather.c"),
    ("ref_coarse", "PyOpenCL27C/Pipe/coarse.c"),
    ("ref_draw", "PyOpenCL27C/Shaders/drawtexcolsmp.c"),
    ("ref_draw_alpha", "PyOpenCL27C/Shaders/drawtexcolsmpalpha.c"),
    ("ref_drawmin", "PyOpenCL27C/Shaders/drawmin.c"),
    ("ref_drawmin_alpha", "PyOpenCL27C/Shaders/drawminalpha.c"),
    ("ref_clearzb", "PyOpenCL27C/Shaders/clearzb.c"),
    ("ref_gamma", "PyOpenCL27C/Shaders/Post/gamma.c"),
    ("ref_vert", "PyOpenCL27C/Pipe/vert.c"),
    ("ref_ssao", "PyOpenCL27C/Shaders/Post/ssao.c"),
    ("ref_dof", "PyOpenCL27C/Shaders/Post/dof.c"),
    ("ref_blur", "PyOpenCL27C/Shaders/Post/blur.c"),
    ("ref_blur2", "PyOpenCL27C/Shaders/Post/blur2.c"),
    # the 4-way blend stores `convert_ushort(blend) * light` into u16 planes
    ("ref_drawmulti", "PyOpenCL27C/Shaders/drawmulti.c", SAT_STORES),
]

# kernels the reference generates from an AVSL source with its own
# Shaders_src/AVSL.py (compile_AVSL: the tiled `draw`, then `drawSmall`, as
# compile_file writes them): (namespace, AVSL source, prelude).  The
# normal-mapped materials call `sampleShadow`, which the reference defines
# nowhere; the prelude defines it as this library does (its own choice):
# the five taps of one cascade (centre, +-2 texels in x and y) at the
# truncated map position, counted where the map is nearer than `depth`,
# only when the centre lies in [2, 2 wS - 2) on both axes; the shadowed
# fraction is count * 0.2.
SHADOW5 = """
inline float sampleShadow(float depth, float sfx, float sfy, float *SD, int wS, float) {
  int sx = cvt_int(sfx), sy = cvt_int(sfy), n = 0;
  if (sx >= 2 && sx < 2 * wS - 2 && sy >= 2 && sy < 2 * wS - 2) {
    if (SD[2 * wS * sy + sx] < depth) n += 1;
    if (SD[2 * wS * (sy + 2) + sx] < depth) n += 1;
    if (SD[2 * wS * (sy - 2) + sx] < depth) n += 1;
    if (SD[2 * wS * sy + (sx + 2)] < depth) n += 1;
    if (SD[2 * wS * sy + (sx - 2)] < depth) n += 1;
  }
  return (float)n * 0.2f;
}
"""
GENERATED = [
    ("ref_draw_mip", "PyOpenCL27C/Shaders_src/av_draw_normmap_mip.c", SHADOW5),
    ("ref_draw_nrm", "PyOpenCL27C/Shaders_src/av_draw_normmap.c", SHADOW5),
    ("ref_draw_nrm_alpha", "PyOpenCL27C/Shaders_src/av_draw_normmap_alpha.c", SHADOW5),
]

CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math",
            "-fopenmp", "-pthread", "-w", "-DBLOCK_SIZE=128"]

_VEC_LIT = re.compile(r"\((float|int|ushort|uchar)([234])\)\s*\(")
_LOCAL_DECL = re.compile(r"__local\s+(\w+)\s+(\w+)\s*(\[[^\]]*\])?\s*;")


def translate(src: str, ns: str, prelude: str = "") -> str:
    """Mechanical OpenCL C -> C++ rewrite of one kernel file."""
    locals_ = _LOCAL_DECL.findall(src)
    body = _VEC_LIT.sub(lambda m: f"make_{m.group(1)}{m.group(2)}(", src)
    body = _LOCAL_DECL.sub(lambda m: f"extern thread_local {m.group(1)} {m.group(2)}{m.group(3) or ''};", body)
    body = re.sub(r"\b__kernel\b", "", body)
    body = re.sub(r"\b__global\b", "", body)
    body = re.sub(r"\b__constant\b", "", body)
    defs = "".join(f"thread_local {t} {n}{dim};\n" for t, n, dim in locals_)
    getters = ""
    for t, n, dim in locals_:
        getters += f"{t} *local_{n}() {{ return {'' if dim else '&'}{n}; }}\n"
    return (f'#include "ref_shim.h"\nnamespace cl_shim {{ namespace {ns} {{\n{prelude}\n'
            f"{body}\n{defs}{getters}}} }}\n")


# where this recipe reads the reference checkout (read-only; nothing is copied)
DEFAULT_REFERENCE = os.environ.get("AXR_REFERENCE", "/root/reference")


def avsl_expand(reference: str, rel: str) -> str:
    """The OpenCL C the reference's generator makes from an AVSL source (run
    in memory: Shaders_src is imported from the checkout as a package)."""
    root = os.path.join(reference, "PyOpenCL27C")
    sys.path.insert(0, root)
    try:
        import importlib
        avsl = importlib.import_module("Shaders_src.AVSL")
        with open(os.path.join(reference, rel)) as f:
            lines = f.readlines()
        return avsl.compile_AVSL(lines, True) + "\n\n\n" + avsl.compile_AVSL(lines, False)
    finally:
        sys.path.remove(root)
        for k in [k for k in sys.modules if k == "Shaders_src" or k.startswith("Shaders_src.")]:
            del sys.modules[k]


def build(reference: str = DEFAULT_REFERENCE, verbose: bool = False) -> str | None:
    if not os.path.isdir(os.path.join(reference, "PyOpenCL27C")):
        print(f"build_ref: reference checkout not found at {reference}; skipped")
        return None
    os.makedirs(OUT, exist_ok=True)
    objs = []
    for ns, rel, *pre in KERNELS:
        path = os.path.join(reference, rel)
        with open(path) as f:
            src = translate(f.read(), ns, pre[0] if pre else "")
        obj = os.path.join(OUT, ns + ".o")
        cmd = ["g++", *CXXFLAGS, "-I", HERE, "-x", "c++", "-c", "-", "-o", obj]
        if verbose:
            print(" ".join(cmd), "<", rel)
        subprocess.run(cmd, input=src.encode(), check=True)
        objs.append(obj)
    for ns, rel, pre in GENERATED:
        src = translate(avsl_expand(reference, rel), ns, pre)
        obj = os.path.join(OUT, ns + ".o")
        cmd = ["g++", *CXXFLAGS, "-I", HERE, "-x", "c++", "-c", "-", "-o", obj]
        if verbose:
            print(" ".join(cmd), "<", rel, "(expanded)")
        subprocess.run(cmd, input=src.encode(), check=True)
        objs.append(obj)
    harness = os.path.join(HERE, "ref_harness.cpp")
    hobj = os.path.join(OUT, "ref_harness.o")
    subprocess.run(["g++", *CXXFLAGS, "-I", HERE, "-c", harness, "-o", hobj], check=True)
    subprocess.run(["g++", "-shared", "-fopenmp", "-pthread", "-o", LIB, hobj, *objs], check=True)
    return LIB


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REFERENCE)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    lib = build(a.reference, a.verbose)
    if lib:
        print("built", lib)
    return 0


if __name__ == "__main__":
    sys.exit(main())
