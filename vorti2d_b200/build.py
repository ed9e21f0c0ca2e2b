"""Build libvorti2d_b200.so in-tree with nvcc for sm_100a.

Usage: python -m vorti2d_b200.build [--force]

Translation units that evaluate the reference's metric / assembly arithmetic
are compiled with -fmad=false, so their results are bit-identical to the CPU
restatement; the Krylov units keep FMA contraction.
"""
from __future__ import annotations

import hashlib
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
    ("v2d_shape.cu", ["-fmad=false"]),
    ("v2d_batch.cu", []),
]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build vorti2d_b200")


def _digest(paths: list[str], flags: list[str]) -> str:
    """Content hash of the inputs of one build step (file contents and flags,
    not modification times: a prebuilt file copied next to changed sources
    with a newer time stamp must still be rebuilt)."""
    h = hashlib.sha256()
    root = os.path.dirname(HERE)
    for f in flags:   # paths relative to the checkout, which moves between machines
        f = os.path.relpath(f, root) if os.path.isabs(f) else f
        h.update(f.encode() + b"\0")
    for p in sorted(paths):
        h.update(os.path.basename(p).encode() + b"\0")
        with open(p, "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()


def _stale(target: str, digest: str) -> bool:
    """True unless target exists and its stamp file records this digest."""
    stamp = target + ".sha256"
    if not (os.path.exists(target) and os.path.exists(stamp)):
        return True
    with open(stamp) as fh:
        return fh.read().strip() != digest


def _stamp(target: str, digest: str) -> None:
    with open(target + ".sha256", "w") as fh:
        fh.write(digest + "\n")


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
        cmd = [nv, *ARCH, *COMMON, *extra, "-c", path, "-o", obj]
        dg = _digest([path] + headers, cmd[1:])
        if force or _stale(obj, dg):
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.check_call(cmd)
            _stamp(obj, dg)
    cmd = [nv, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    dg = _digest(objs, cmd[1:])
    if force or _stale(LIB, dg):
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        _stamp(LIB, dg)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
