"""Build recipe for the engine's shared library (``libdfem.so``, in-tree).

nvcc cross-compiles for sm_100a only; the host C++ (ordering, symbolic and
numeric factorisation, scene preprocessing) is compiled by nvcc's host
compiler into the same library.  ``python -m diff_fem_b200.build`` rebuilds it.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libdfem.so")
SOURCES = ["engine.cu", "noalloc.cu", "scene.cpp", "cholesky.cpp", "resident_plan.cpp", "obj_writer.cpp"]
HEADERS = ["pd_kernels.cu", "pd_math.cuh", "kernels.cuh", "factor_kernels.cuh", "contact_kernels.cuh", "tma.cuh",
           "resident_solve.cuh", "drag_kernels.cuh", "skeleton_kernels.cuh", "skeleton_adjoint.cuh", "dense_solve.cuh",
           "scene.h", "cholesky.h", "resident_plan.h"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-O3",
    "-shared",
]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "dfem.h"))
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    cmd = [NVCC, *NVCC_FLAGS, "-o", LIB + ".tmp", *[os.path.join(CSRC, f) for f in SOURCES]]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
