"""Build libanacapa_b200.so in-tree for sm_100a.

    python -m anacapa_b200.build [--force]

The CUDA kernels are compiled with nvcc for sm_100a only; the host scene
preparation is compiled with -ffp-contract=off (every float operation rounds
on its own, matching the reference's float code op for op).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "libanacapa_b200.so")

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
CUDA_HOME = os.path.dirname(os.path.dirname(os.path.realpath(NVCC)))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

SOURCES = {
    "kernels.cu": ["kernels.cu", "kernels.h", "layout.h", "dmath.cuh", "sampler.cuh", "shade.cuh",
                   "traverse.cuh", "motion.cuh"],
    "build.cu": ["build.cu", "build.h", "layout.h"],
    "prepare.cpp": ["prepare.cpp", "prepare.h", "layout.h"],
    "capi.cpp": ["capi.cpp", "kernels.h", "prepare.h", "build.h", "layout.h"],
    "film_io.cpp": ["film_io.cpp"],
}


def _newer(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    hdr = os.path.join(ROOT, "include", "anacapa_b200.h")
    return any(os.path.getmtime(os.path.join(CSRC, d)) > t for d in deps) or os.path.getmtime(hdr) > t


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force=False, verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    rebuilt = False
    inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
    for src, deps in SOURCES.items():
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if not force and not _newer(obj, deps):
            continue
        rebuilt = True
        path = os.path.join(CSRC, src)
        if src.endswith(".cu"):
            cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                   "--expt-relaxed-constexpr", *inc, "-c", path, "-o", obj]
            if src == "build.cu":  # every float operation rounds on its own
                cmd.insert(1, "-fmad=false")
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
        else:
            flags = ["-O2", "-std=c++17", "-fPIC", "-pthread", f"-I{CUDA_HOME}/include", *inc]
            if src == "prepare.cpp":
                flags.append("-ffp-contract=off")
            cmd = [os.environ.get("CXX", "g++"), *flags, "-c", path, "-o", obj]
        _run(cmd, verbose)
    if rebuilt or force or not os.path.exists(LIB):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lpthread", "-lz"], verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
