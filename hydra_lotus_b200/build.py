"""Builds the CUDA library (hydra_lotus_b200/_lib/liblotus_cuda.so) with
nvcc for sm_100a.

The library is compiled with --fmad=false so that the transport's multiply
and add steps round separately in source order.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIB_DIR, "liblotus_cuda.so")
INCLUDE = os.path.join(HERE, "..", "include")
SOURCES = ["integrator.cu", "bvh_build.cu", "renderer.cu", "static_render.cu", "temporal.cu",
           "radiance_cache.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-Wall"]


def _inputs():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)
             if f.endswith((".cu", ".cuh", ".h"))]
    files += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return files


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in _inputs())


def build(force=False, verbose=False, jobs=None):
    """Compiles each source to an object in parallel, then links."""
    if not force and not stale():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    objs = []
    procs = []
    for src in SOURCES:
        obj = os.path.join(LIB_DIR, src.replace(".cu", ".o"))
        cmd = ["nvcc"] + ARCH + FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append(subprocess.Popen(cmd))
        objs.append(obj)
    for p in procs:
        if p.wait() != 0:
            raise RuntimeError("nvcc failed")
    cmd = ["nvcc"] + ARCH + ["-shared", "-o", LIB] + objs
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
