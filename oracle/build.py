"""Builds the oracle (test infrastructure only) into oracle/_build/:

* liboracle.so   -- the CPU restatement of the numeric phase (oracle.cpp);
* libanalysis.so -- the library's host analysis (symbolic analysis and MC64
  from rivrs-linalg_b200/csrc) without the CUDA numeric phase, for processes
  that run the CPU restatement alone (analysis_shim.cpp).

    python oracle/build.py

-ffp-contract=off keeps every unfused expression unfused; std::fma and the
AVX-512 tile kernel's vfnmadd mark the fused ones (see the arithmetic
contract at the top of oracle.cpp).  -mfma lets std::fma compile to the FMA
instruction instead of a library call; the AVX-512 kernel is compiled for
that target alone and chosen at run time.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "liboracle.so")
SRC = os.path.join(HERE, "oracle.cpp")
ALIB = os.path.join(OUT, "libanalysis.so")
CSRC = os.path.join(ROOT, "rivrs-linalg_b200", "csrc")
ASRC = [os.path.join(HERE, "analysis_shim.cpp")] + [os.path.join(CSRC, f) for f in
                                                    ("symbolic.cpp", "capi.cpp", "mc64.cpp")]
ADEPS = ASRC + [os.path.join(CSRC, "rvg_internal.h"), os.path.join(ROOT, "include", "rivrs_b200.h")]


def _stale(out, deps):
    return not os.path.exists(out) or any(os.path.getmtime(d) > os.path.getmtime(out) for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("oracle build failed: " + os.path.basename(cmd[-1]))


def build(verbose=False):
    os.makedirs(OUT, exist_ok=True)
    if _stale(LIB, [SRC]):
        _run(["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-mfma",
              "-o", LIB, SRC])
    if _stale(ALIB, ADEPS):
        _run(["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off",
              "-I", os.path.join(ROOT, "include"), "-o", ALIB] + ASRC)
    if verbose:
        print("built", LIB, ALIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
