"""Builds the engine's shared library in-tree with nvcc for sm_100a.

The kernels are instantiated in one translation unit per (compute type, e-e-n order), compiled
in parallel with the C-ABI unit and the host-side linear-method unit, then linked into
libchamp_b200.so.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
UNITS = ["host.cu", "linear.cu", "optimize.cu", "tune.cu"] + [f"inst_{t}_n{n}.cu" for t in ("f32", "f64") for n in (0, 4, 5)]
DEPS = [os.path.join(HERE, "..", "include", "champ_b200.h")] + glob.glob(os.path.join(CSRC, "*"))
LIB = os.path.join(HERE, "libchamp_b200.so")
OBJDIR = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in DEPS)


def build(force: bool = False, verbose: bool = False) -> str:
    if not (force or needs_build()):
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)

    def compile_unit(u):
        obj = os.path.join(OBJDIR, u.replace(".cu", ".o"))
        cmd = [NVCC] + FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-c", os.path.join(CSRC, u), "-o", obj]
        subprocess.check_call(cmd)
        return obj

    with ThreadPoolExecutor(len(UNITS)) as ex:
        objs = list(ex.map(compile_unit, UNITS))
    subprocess.check_call([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcublas"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
