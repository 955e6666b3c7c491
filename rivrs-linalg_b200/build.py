"""Builds the in-tree shared library `librivrs_b200.so` for sm_100a.

    python rivrs-linalg_b200/build.py

CUDA sources are compiled with `-gencode arch=compute_100a,code=sm_100a` and
`--fmad=false`: the kernels place every fused multiply-add explicitly
(`__fma_rn`) where the arithmetic contract calls for one, and nothing else
may be contracted.  Host C++ is compiled with `-ffp-contract=off` for the
same reason.  The selector network's training kernels (`mlp.cu`: forward for
prediction, gradient, Adam) have no bit-for-bit contract (they are checked
against a float64 oracle within tolerances), so they are compiled with
`--fmad=true`; the network's inference during a factorization is part of
`numeric.cu` and keeps the contract.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "librivrs_b200.so")
BUILD = os.path.join(HERE, "_build")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
            "-I", os.path.join(ROOT, "include")] + ARCH
CU_FMAD = {"mlp.cu": True}  # sources without the exact-arithmetic contract (default: --fmad=false)
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I", os.path.join(ROOT, "include")]

CU_SOURCES = ["numeric.cu", "noalloc.cu", "mlp.cu"]
CXX_SOURCES = ["symbolic.cpp", "plan.cpp", "capi.cpp", "mc64.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + os.path.basename(cmd[-1]))
    return r


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "rivrs_b200.h"))
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if _stale(o, [s] + headers + [os.path.abspath(__file__)]):
            fmad = "--fmad=true" if CU_FMAD.get(src) else "--fmad=false"
            _run([NVCC] + CU_FLAGS + [fmad, "-c", s, "-o", o])
        objs.append(o)
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if _stale(o, [s] + headers):
            _run(["g++"] + CXX_FLAGS + ["-c", s, "-o", o])
        objs.append(o)
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
