"""Build libfastgpr.so (and its bounds-checked twin) in-tree for sm_100a.

    python fast-gpr-fwi_b200/build.py [--force]

The shared objects land in fast-gpr-fwi_b200/_lib/ so they travel with the
source tree; nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "_lib")
SOURCES = [os.path.join(CSRC, "fastgpr.cu")]
DEPS = SOURCES + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")] + [
    os.path.join(HERE, "..", "include", "fastgpr.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    # no implicit FMA contraction: every fused multiply-add is explicit
    "-fmad=false",
    "-Xcompiler", "-fPIC", "-shared",
]

TARGETS = {
    "libfastgpr.so": [],
    "libfastgpr_checked.so": ["-DFG_CHECKED"],
}


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _stale(target: str) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in DEPS if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> list:
    os.makedirs(LIB_DIR, exist_ok=True)
    jobs = []
    for name, extra in TARGETS.items():
        out = os.path.join(LIB_DIR, name)
        if not force and not _stale(out):
            continue
        cmd = [_nvcc()] + NVCC_FLAGS + extra + ["-o", out] + SOURCES
        if verbose:
            print(" ".join(cmd), flush=True)
        jobs.append((out, cmd, subprocess.Popen(cmd)))
    for out, cmd, proc in jobs:
        if proc.wait() != 0:
            raise subprocess.CalledProcessError(proc.returncode, cmd)
    return [out for out, _, _ in jobs]


if __name__ == "__main__":
    force = "--force" in sys.argv
    for p in build(force=force, verbose=True):
        print("built", p)
