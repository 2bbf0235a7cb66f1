"""Build the in-tree CUDA library ``pargemslr_b200/_lib/libpgx.so`` for sm_100a.

    python -m pargemslr_b200.build

nvcc cross-compiles for Blackwell (sm_100a) without a GPU present; the
resulting shared object is loaded by :mod:`pargemslr_b200._abi` through ctypes
and exports exactly the C ABI declared in ``include/pgx.h``.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libpgx.so")
SOURCES = [os.path.join(CSRC, "pgx.cu"), os.path.join(CSRC, "setup.cpp"), os.path.join(CSRC, "params.cpp"),
           os.path.join(CSRC, "hypre.cpp")]
HEADERS = [os.path.join(CSRC, "pgx_device.cuh"), os.path.join(CSRC, "pgx_complex.cuh"), os.path.join(CSRC, "pgx_umma.cuh"), os.path.join(CSRC, "pgx_systems.cuh"), os.path.join(CSRC, "pgx_setup.h"), os.path.join(CSRC, "pgx_params.h"),
           os.path.join(CSRC, "pgx_internal.h"), os.path.join(ROOT, "include", "pgx_hypre.h"),
           os.path.join(ROOT, "include", "pgx.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", "-Xcompiler", "-fopenmp",
    "-shared", "-lgomp",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *NVCC_FLAGS, "-o", tmp, *SOURCES]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
