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
# (source, extra flags): the FP64 parity form reproduces the reference's IEEE
# operation order (no FMA contraction, IEEE division and square root); the
# mixed form (FP32 fluxes) is compiled with contraction and fast FP32 division.
FP64_FLAGS = ["-fmad=false", "-prec-div=true", "-prec-sqrt=true"]
MIXED_FLAGS = ["-fmad=true", "-prec-div=false", "-prec-sqrt=false"]
_C = os.path.join(PKG_DIR, "csrc")
# (source, flags, object name): cb_stage_parts.cu is compiled once per form
# (FP64 / mixed), LES value and launch kind (single block / batched) so the
# stage-kernel template variants build in parallel
SOURCES = [
    (os.path.join(_C, "cb_api.cu"), FP64_FLAGS, "cb_api"),
    (os.path.join(_C, "cb_noalloc.cu"), FP64_FLAGS, "cb_noalloc"),
    (os.path.join(_C, "cb_batch.cu"), FP64_FLAGS, "cb_batch"),
    (os.path.join(_C, "cb_mixed.cu"), MIXED_FLAGS, "cb_mixed"),
    (os.path.join(_C, "cb_peaks.cu"), FP64_FLAGS, "cb_peaks"),
] + [
    (os.path.join(_C, "cb_stage_parts.cu"),
     (MIXED_FLAGS if mix else FP64_FLAGS) + [f"-DCB_PART_MIX={mix}", f"-DCB_PART_LES={les}", f"-DCB_PART_BATCH={bat}"],
     f"cb_stage_{'mixed' if mix else 'fp64'}_{'les' if les else 'std'}{'_batch' if bat else ''}")
    for mix in (0, 1) for les in (1, 0) for bat in (0, 1)
]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
]


def _deps():
    return (glob.glob(os.path.join(PKG_DIR, "csrc", "*")) + [os.path.join(REPO, "include", "chimera_b200.h")])


def needs_build() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    return any(os.path.getmtime(p) > t for p in _deps())


def _run(cmd, verbose):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libchimera_b200.so: " + " ".join(cmd))
    if verbose:
        sys.stderr.write(r.stderr)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB_PATH
    objdir = os.path.join(PKG_DIR, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs, cmds = [], []
    for src, flags, name in SOURCES:
        obj = os.path.join(objdir, name + ".o")
        cmds.append([NVCC] + NVCC_FLAGS + flags + (["-Xptxas", "-v"] if verbose else []) + ["-c", "-o", obj, src])
        objs.append(obj)
    # the translation units compile in parallel, at most one per core
    failed = None
    jobs = max(1, min(len(cmds), os.cpu_count() or 1))
    pending, running = list(cmds), []
    while pending or running:
        while pending and len(running) < jobs:
            cmd = pending.pop(0)
            running.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
        cmd, p = running.pop(0)
        out, err = p.communicate()
        if p.returncode != 0:
            sys.stderr.write(out + err)
            failed = failed or cmd
        elif verbose:
            sys.stderr.write(err)
    if failed:
        raise RuntimeError("nvcc failed building libchimera_b200.so: " + " ".join(failed))
    _run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB_PATH] + objs, verbose)
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB_PATH)
