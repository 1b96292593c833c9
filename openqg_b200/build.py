"""Build recipe of the CUDA library (sm_100a) and loader of its path.

`python -m openqg_b200.build` compiles openqg_b200/csrc into
openqg_b200/liboqg.so with nvcc for sm_100a.  The library is built in-tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "liboqg.so")
SOURCES = ["oqg_capi.cu", "oqg_setup.cpp", "oqg_radiat.cpp"]
DEPS = SOURCES + ["oqg_dev.cuh", "oqg_fft.cuh", "oqg_kernels.cuh", "oqg_tma.cuh", "oqg_setup.h",
                  "oqg_adjoint.cuh", "oqg_noalloc.cuh", "oqg_mixed.cuh",
                  os.path.join("..", "..", "include", "oqg.h")]

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
    "-ccbin", "/usr/bin/g++",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(os.path.join(CSRC, d)) > t for d in DEPS)


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    if not force and not stale():
        return LIB
    cmd = [nvcc()] + NVCC_FLAGS + (extra or []) + ["-shared", "-o", LIB] + \
          [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building %s" % LIB)
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None)
