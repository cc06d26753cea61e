"""Builds the in-tree CUDA library crava_b200/lib/libcrava_gpu.so for sm_100a.

Each translation unit is compiled with
  nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3
and linked into one shared library with a static CUDA runtime.  The files
that must round like the reference's FP32 code (solve_ref.cu, sim.cu) are
compiled with -fmad=false.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libcrava_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = {
    "capi.cu": [],
    "fft.cu": [],
    "cols_tma.cu": [],
    "plane.cu": [],
    "solve.cu": [],
    "solve_ref.cu": ["-fmad=false"],
    "sim.cu": ["-fmad=false"],
    "unit.cu": [],
    "noalloc.cu": [],
    "batch.cu": [],
    "loglik.cu": [],
    "forward.cu": [],
    "prior.cu": [],
    "crava_file.cu": [],
    "state4d.cu": ["-fmad=false"],
    "divide.cu": [],
    "interp.cu": [],
}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, extra=()) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "crava_gpu.h"))
    objs = []
    for src, flags in SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _newer(o, [s] + headers):
            cmd = [NVCC, *ARCH, *FLAGS, *flags, *extra, "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _newer(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
