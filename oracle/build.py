"""Builds the oracle (test infrastructure only) into oracle/_build/liboracle.so.

    python oracle/build.py

-ffp-contract=off keeps every unfused expression unfused; std::fma marks the
fused ones (see the arithmetic contract at the top of oracle.cpp).  -mfma
lets std::fma compile to the FMA instruction instead of a library call.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "liboracle.so")
SRC = os.path.join(HERE, "oracle.cpp")


def build(verbose=False):
    os.makedirs(OUT, exist_ok=True)
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-mfma",
           "-o", LIB, SRC]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("oracle build failed")
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
