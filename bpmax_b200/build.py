"""Builds bpmax_b200/libbpmax_gpu.so in-tree with nvcc for sm_100a (no JIT, no torch).

    python -m bpmax_b200.build          # or bpmax_b200.build.build()
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libbpmax_gpu.so")

SOURCES = ["bpmax_engine.cu", "bpmax_shim.cpp"]
HEADERS = ["bpmax_kernels.cuh", "bpmax_kernels_large.cuh", "bpmax_r0.cuh", "bpmax_adjoint.cuh", "bpmax_r0only.cuh",
           "bpmax_wide.cuh", "bpmax_persist.cuh", "r0_tables.inc", "wide_tables.inc"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-O2", "-shared",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "bpmax_gpu.h")]
    return any(os.path.getmtime(p) > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    srcs = [os.path.join(CSRC, f) for f in SOURCES]
    cmd = [nvcc(), *NVCC_FLAGS, "-Xptxas", "-v" if verbose else "-O3", "-o", LIB + ".tmp", *srcs]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError("nvcc failed building libbpmax_gpu.so")
    if verbose:
        sys.stderr.write(proc.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
