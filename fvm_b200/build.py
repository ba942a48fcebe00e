"""Builds fvm_b200/libfvm_b200.so (host C++ + sm_100a CUDA) in place.

    python -m fvm_b200.build          # or fvm_b200.build.build()

Objects go to fvm_b200/_build; the shared library sits next to this file so
that it travels with the source tree. Host code is compiled with
-ffp-contract=off and device code with -fmad=false: the mesh geometry,
matrix coefficients and AMG setup must round exactly like the reference's
scalar C++ for the integer setup (aggregation) to match it bit for bit.
Files whose results need no bitwise match with the reference (the learned
network, the GPU-built hierarchy of the mixed-precision path) are compiled
with fused multiply-adds (FMA_SOURCES).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfvm_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-function"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC,-ffp-contract=off"] + ARCH

HOST_SOURCES = ["mesh.cpp", "amg_setup.cpp", "capi.cpp", "fluent.cpp"]
CUDA_SOURCES = ["kernels.cu", "solver.cu", "thermal.cu", "residual_noalloc.cu", "learned.cu", "amg_device.cu"]
# device code free to contract a * b + c into one rounding
FMA_SOURCES = {"learned.cu", "amg_device.cu"}


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _cuda_home() -> str:
    return os.path.dirname(os.path.dirname(os.path.realpath(_nvcc())))


def _newer(src_list, target) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_list)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    hs.append(os.path.join(ROOT, "include", "fvm_b200.h"))
    return hs


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    nvcc = _nvcc()
    inc = ["-I" + CSRC, "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(_cuda_home(), "include")]
    headers = _headers()
    jobs = []
    objs = []
    for f in HOST_SOURCES:
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJ, f + ".o")
        objs.append(obj)
        if force or _newer([src] + headers, obj):
            jobs.append(["g++"] + CXX_FLAGS + inc + ["-c", src, "-o", obj])
    for f in CUDA_SOURCES:
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJ, f + ".o")
        objs.append(obj)
        if force or _newer([src] + headers, obj):
            fmad = ["-fmad=true"] if f in FMA_SOURCES else ["-fmad=false"]
            jobs.append([nvcc] + NVCC_FLAGS + fmad + inc + ["-c", src, "-o", obj])
    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for out in ex.map(_run, jobs):
            if verbose and out.strip():
                print(out)
    if force or _newer(objs, LIB):
        _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-ldl"])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
