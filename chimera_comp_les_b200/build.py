"""Builds libchimera_b200.so in-tree with nvcc for sm_100a.

The shared library is the product: CUDA kernels plus the C-ABI declared in
include/chimera_b200.h.  It is rebuilt when any source is newer than it.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG_DIR)
LIB_PATH = os.path.join(PKG_DIR, "libchimera_b200.so")
SOURCES = [os.path.join(PKG_DIR, "csrc", "cb_api.cu"), os.path.join(PKG_DIR, "csrc", "cb_noalloc.cu")]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
# The FP64 form reproduces the reference's IEEE operation order: no FMA
# contraction (-fmad=false), IEEE division and square root.
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC", "-shared",
]


def _deps():
    return (glob.glob(os.path.join(PKG_DIR, "csrc", "*")) + [os.path.join(REPO, "include", "chimera_b200.h")])


def needs_build() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    return any(os.path.getmtime(p) > t for p in _deps())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB_PATH
    cmd = [NVCC] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-o", LIB_PATH] + SOURCES
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libchimera_b200.so")
    if verbose:
        sys.stderr.write(r.stderr)
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB_PATH)
