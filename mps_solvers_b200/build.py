"""Build libmps_b200.so in-tree with nvcc for sm_100a.

    python -m mps_solvers_b200.build            # incremental
    python -m mps_solvers_b200.build --force    # rebuild everything

The library is plain CUDA runtime + C++ (no torch); it is loaded with ctypes
by mps_solvers_b200.capi and can be linked by any C/C++ caller through
include/mps_capi.h.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmps_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOSTCXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false is not used: the exact kernels use explicit _rn intrinsics and
# the fast kernels are allowed to contract.
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
                  "-ccbin", HOSTCXX, "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]
CXXFLAGS = ["-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", "-fno-fast-math",
            "-I/usr/local/cuda/include"]

CU = ["cellsort.cu", "physics.cu", "ppe.cu", "ppe_compact.cu", "learned.cu", "surface.cu", "capi.cu", "noalloc.cu"]
CPP = ["host_io.cpp"]


def _deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(HERE, "..", "include", "mps_capi.h")]


def _stale(obj, src):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in _deps() + [src])


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    jobs = []
    objs = []
    for f in CU:
        src, obj = os.path.join(CSRC, f), os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            jobs.append([NVCC] + NVFLAGS + ["-c", src, "-o", obj])
    for f in CPP:
        src, obj = os.path.join(CSRC, f), os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            jobs.append([HOSTCXX] + CXXFLAGS + ["-c", src, "-o", obj])
    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        outs = list(ex.map(_run, jobs))
    if verbose:
        for o in outs:
            if o.strip():
                print(o)
    if jobs or force or not os.path.exists(LIB):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
