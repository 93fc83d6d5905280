"""Build the native library ``libfribois2d.so`` in-tree with nvcc (sm_100a).

No PyTorch or JIT cache is involved: the shared library sits next to this
file so that it travels with the source tree.  Usage::

    python -m fribois2d_b200.build [--force]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "libfribois2d.so")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false keeps every FP64 expression unfused, as the reference's
# -O3 -msse2 build evaluates it; the line-solve and GEMM units opt back in.
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp,-ffp-contract=off",
          f"-I{INCLUDE}", f"-I{CSRC}"]
UNITS = [
    ("host.cpp", ["-fmad=false"]),
    ("kernels.cu", ["-fmad=false"]),
    ("tri.cu", []),
    ("tc_gemm.cu", []),
    ("mlp.cu", []),
    ("couple.cu", ["-fmad=false"]),
    ("api.cu", ["-fmad=false"]),
    ("noalloc.cu", ["-fmad=false"]),
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _sources():
    out = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".cu", ".cuh", ".cpp", ".h")):
            out.append(os.path.join(CSRC, f))
    out.append(os.path.join(INCLUDE, "fribois2d.h"))
    return out


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in _sources())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    objs, cmds = [], []
    for src, extra in UNITS:
        obj = os.path.join(BUILD, src + ".o")
        cmds.append([nvcc, *ARCH, *COMMON, *extra, "-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    # the units compile independently: one nvcc per unit, in parallel
    from concurrent.futures import ThreadPoolExecutor
    if verbose:
        for cmd in cmds:
            print(" ".join(cmd))
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
        for _ in ex.map(subprocess.check_call, cmds):
            pass
    tmp = LIB + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-o", tmp, *objs, "-lcublas", "-lcublasLt", "-lgomp", "-Xcompiler", "-fPIC"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
