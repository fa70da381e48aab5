"""Builds the in-tree shared library ``mr3smp_b200/lib/libmr3b200.so``.

The CUDA layer (``csrc/solver.cu``) is compiled for sm_100a only, with
``-fmad=false`` so that no multiply-add is contracted: every recurrence keeps
the IEEE double arithmetic of the reference's Fortran kernels.  The C host
library (``csrc/mrrr.c``) is compiled with gcc.  The CUDA runtime is linked
statically so the library loads on any box with the driver.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libmr3b200.so")
BUILD = os.path.join(HERE, "_build")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC", "-I" + INC,
    "-diag-suppress", "550,177",
]
CC_FLAGS = ["-O2", "-std=gnu11", "-fPIC", "-Wall", "-I" + INC]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))
            if f.endswith((".cu", ".c", ".cuh", ".h"))] + \
           [os.path.join(INC, f) for f in os.listdir(INC) if f.endswith(".h")]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in _sources())


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile and link the library if any source is newer; returns its path."""
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    nvcc = _nvcc()
    objs = []
    for f in sorted(os.listdir(CSRC)):
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        if f.endswith(".cu"):
            cmd = [nvcc, *NVCC_FLAGS, "-c", src, "-o", obj]
        elif f.endswith(".c"):
            cmd = ["gcc", *CC_FLAGS, "-c", src, "-o", obj]
        else:
            continue
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc, "-shared", "-cudart", "static", "-Wno-deprecated-gpu-targets", "-o", tmp, *objs,
           "-lpthread", "-ldl"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
