"""Build libvorti2d_b200.so in-tree with nvcc for sm_100a.

Usage: python -m vorti2d_b200.build [--force]

Translation units that evaluate the reference's metric / assembly arithmetic
are compiled with -fmad=false, so their results are bit-identical to the CPU
restatement; the Krylov units keep FMA contraction.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libvorti2d_b200.so")

# (source, extra flags)
SOURCES = [
    ("v2d_util.cu", []),
    ("v2d_seam.cu", ["-fmad=false"]),
    ("v2d_assemble.cu", ["-fmad=false"]),
    ("v2d_krylov.cu", []),
    ("v2d_mf.cu", []),
    ("v2d_solver.cu", []),
    ("v2d_forces.cu", []),
    ("v2d_velocity.cu", ["-fmad=false"]),
    ("v2d_linsys.cu", []),
]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build vorti2d_b200")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(INCLUDE, "vorti2d_b200.h"))
    objs = []
    nv = nvcc()
    for src, extra in SOURCES:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(OUT_DIR, src.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [path, __file__] + headers):
            cmd = [nv, *ARCH, *COMMON, *extra, "-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.check_call(cmd)
    if force or _stale(LIB, objs):
        cmd = [nv, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
