"""Build libuwshcu_b200.so in-tree with nvcc for sm_100a.

Each .cu translation unit is compiled to an object under _build/ and the objects are linked into
lib/libuwshcu_b200.so (the CUDA runtime is linked statically, nvcc's default).  The FP64 kernel TU
is compiled with -fmad=false so no multiply-add is contracted into an FMA: every operation rounds
as the Fortran writes it.  A unit is rebuilt when its source or any header under csrc/ or include/
is newer than its object.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(REPO, "include")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libuwshcu_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "-I", CSRC, "-I", INCLUDE]
UNITS = {
    "uwshcu_fp64_k32n5.cu": ["-fmad=false"],
    "uwshcu_fp64_k64n5.cu": ["-fmad=false"],
    "uwshcu_fp64_k32n32.cu": ["-fmad=false"],
    "uwshcu_fp64_k64n32.cu": ["-fmad=false"],
    # the fast-FP64 mode is not bit-exact by design: FMA contraction allowed
    "uwshcu_fast_k32n5.cu": [],
    "uwshcu_fast_k64n5.cu": [],
    "uwshcu_fast_k32n32.cu": [],
    "uwshcu_fast_k64n32.cu": [],
    "uwshcu_mixed_k32n5.cu": [],
    "uwshcu_mixed_k64n5.cu": [],
    "uwshcu_budget.cu": ["-fmad=false"],
    # tangent-linear kernels: no FMA contraction, so their values are the FP64 path's bits
    "uwshcu_tl_k32n5.cu": ["-fmad=false"],
    "uwshcu_tl_k64n5.cu": ["-fmad=false"],
    # adjoint kernels: no FMA contraction, so their forward values are the FP64 path's bits
    "uwshcu_adj_k32n5.cu": ["-fmad=false"],
    "uwshcu_adj_k64n5.cu": ["-fmad=false"],
    "uwshcu_host.cu": [],
    # measured FP64 throughput (explicit fma: the flag does not matter)
    "uwshcu_probe.cu": [],
}


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def _headers_mtime():
    t = 0.0
    for d in (CSRC, INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".cuh", ".h")):
                t = max(t, os.path.getmtime(os.path.join(d, f)))
    return t


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdr = _headers_mtime()
    objs, relink, jobs = [], force or not os.path.exists(LIB), []
    for unit, flags in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        objs.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr):
            jobs.append([nvcc()] + ARCH + COMMON + flags + ["-c", src, "-o", obj])
    if jobs:
        relink = True
        procs = []
        for cmd in jobs:
            if verbose:
                print(" ".join(cmd), flush=True)
            procs.append(subprocess.Popen(cmd))
        bad = [p.wait() for p in procs]
        if any(bad):
            raise RuntimeError("nvcc failed")
    if relink or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
