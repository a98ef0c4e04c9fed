"""Build libfastgpr.so (and its bounds-checked twin) in-tree for sm_100a.

    python fast-gpr-fwi_b200/build.py [--force] [libfastgpr.so | libfastgpr_checked.so]

Each kernel family is its own translation unit (csrc/*.cu); the units are
compiled in parallel into objects under _build/ and linked into the shared
objects in fast-gpr-fwi_b200/_lib/, so they travel with the source tree;
nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "_lib")
OBJ_DIR = os.path.join(HERE, "_build")
SOURCES = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))
DEPS = SOURCES + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + [
    os.path.join(HERE, "..", "include", "fastgpr.h"), os.path.abspath(__file__)]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-lineinfo", "-O3", "-std=c++17",
    # no implicit FMA contraction: every fused multiply-add is explicit
    "-fmad=false",
    "-Xcompiler", "-fPIC",
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


def _run_all(jobs, verbose):
    procs = []
    for cmd in jobs:
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd)))
    for cmd, proc in procs:
        if proc.wait() != 0:
            raise subprocess.CalledProcessError(proc.returncode, cmd)


def build(force: bool = False, verbose: bool = False, only=None) -> list:
    os.makedirs(LIB_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    todo = [(name, extra) for name, extra in TARGETS.items()
            if (only is None or name in only) and (force or _stale(os.path.join(LIB_DIR, name)))]
    compile_jobs, objects = [], {}
    for name, extra in todo:
        tag = os.path.splitext(name)[0]
        objects[name] = []
        for src in SOURCES:
            obj = os.path.join(OBJ_DIR, "%s.%s.o" % (tag, os.path.splitext(os.path.basename(src))[0]))
            objects[name].append(obj)
            compile_jobs.append([_nvcc()] + NVCC_FLAGS + extra + ["-c", "-o", obj, src])
    _run_all(compile_jobs, verbose)
    link_jobs = [[_nvcc()] + ARCH + ["-shared", "-o", os.path.join(LIB_DIR, name)] + objects[name] for name, _ in todo]
    _run_all(link_jobs, verbose)
    return [os.path.join(LIB_DIR, name) for name, _ in todo]


if __name__ == "__main__":
    force = "--force" in sys.argv
    only = [a for a in sys.argv[1:] if a in TARGETS] or None
    for p in build(force=force, verbose=True, only=only):
        print("built", p)
