"""Builds the oracle's shared library with g++ (TEST INFRASTRUCTURE ONLY).

The oracle is plain FP32 C++: -ffp-contract=off keeps every multiply and
add separately rounded, as the CUDA kernels (built with --fmad=false)
compute them.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liblotus_oracle.so")
SOURCES = [os.path.join(HERE, "lotus_oracle.cpp")]
HEADERS = [os.path.join(HERE, "lotus_oracle.h"),
           os.path.join(HERE, "..", "include", "lotus_cuda.h")]


def stale(target, inputs):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(p) > t for p in inputs)


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    if force or stale(LIB, SOURCES + HEADERS):
        cmd = ["g++", "-O3", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fPIC",
               "-shared", "-Wall", "-Wextra", "-o", LIB] + SOURCES
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
