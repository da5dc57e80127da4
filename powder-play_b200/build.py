"""Builds libmpm_b200.so in-tree with nvcc for sm_100a.

Usage: python powder-play_b200/build.py  (or __graft_entry__.build()).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUTPUT = os.path.join(HERE, "libmpm_b200.so")
SOURCES = ["mpm_kernels.cu", "mpm_solver.cu", "mpm_static_sort.cu", "mpm_adjoint.cu"]
HEADERS = ["mpm_device.cuh", "mpm_kernels.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "-Xptxas", "-v",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for candidate in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if candidate and (os.path.isabs(candidate) and os.path.exists(candidate) or not os.path.isabs(candidate)):
            return candidate
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(OUTPUT):
        return True
    built = os.path.getmtime(OUTPUT)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "mpm_b200.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > built for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return OUTPUT
    cmd = [_nvcc(), *NVCC_FLAGS, "-shared", "-o", OUTPUT + ".tmp",
           *[os.path.join(CSRC, f) for f in SOURCES], "-lcudart"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + proc.stdout + proc.stderr)
    if verbose:
        sys.stderr.write(proc.stderr)
    os.replace(OUTPUT + ".tmp", OUTPUT)
    return OUTPUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
