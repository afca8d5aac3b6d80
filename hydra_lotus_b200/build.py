"""Builds the CUDA library (hydra_lotus_b200/_lib/liblotus_cuda.so) with
nvcc for sm_100a.

The sources whose arithmetic the oracle restates bit for bit (transport,
traversal, ReSTIR, the scene tables) are compiled with --fmad=false, so
that their multiply and add steps round separately in source order. The
radiance cache (checked against its oracle within stated tolerances) and
the BVH builders (whose trees never change a hit: hits are decided by
triangle tests alone) are compiled with fused multiply-adds. The SVGF
passes are not: fused, their edge-stopping and neighbour tests decide
differently from the reference's CPU SVGF at a few pixels a frame.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIB_DIR, "liblotus_cuda.so")
INCLUDE = os.path.join(HERE, "..", "include")
SOURCES = ["integrator.cu", "bvh_build.cu", "renderer.cu", "static_render.cu", "temporal.cu", "svgf.cu",
           "radiance_cache.cu", "batch.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"]
# Sources compiled with fused multiply-adds; every other one with --fmad=false.
FUSED = {"radiance_cache.cu", "bvh_build.cu"}


def _inputs():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)
             if f.endswith((".cu", ".cuh", ".h", ".inc"))]
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
        fmad = ["--fmad=true"] if src in FUSED else ["--fmad=false"]
        cmd = ["nvcc"] + ARCH + FLAGS + fmad + ["-c", os.path.join(CSRC, src), "-o", obj]
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


# The albedo tables' generator (csrc/albedo_tables_gen.cpp), which wrote
# csrc/albedo_tables.inc and checks it: a host program.
TABLE_TOOL = os.path.join(LIB_DIR, "albedo_tables_gen")


def build_table_tool(force=False, verbose=False):
    """Builds the albedo tables' generator; returns its path."""
    src = os.path.join(CSRC, "albedo_tables_gen.cpp")
    inputs = [src, os.path.join(CSRC, "albedo.cuh"), os.path.join(CSRC, "lmath.cuh")]
    if (not force and os.path.exists(TABLE_TOOL) and
            all(os.path.getmtime(p) <= os.path.getmtime(TABLE_TOOL) for p in inputs)):
        return TABLE_TOOL
    os.makedirs(LIB_DIR, exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-ffp-contract=off", src, "-o", TABLE_TOOL, "-lpthread"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return TABLE_TOOL


# The C++ adapter (host/cuda_offscreen_renderer.*) implements the
# reference's Lotus::OffscreenRenderer over the C ABI; it compiles against
# the reference's headers, so it builds only where they are present
# ($LOTUS_REFERENCE, else ../reference beside this checkout). Its test
# driver links it with
# the library into _lib/adapter_harness.
HOST = os.path.join(HERE, "host")
HARNESS = os.path.join(LIB_DIR, "adapter_harness")
REFERENCE = os.environ.get("LOTUS_REFERENCE", os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))


def reference_headers():
    return os.path.exists(os.path.join(REFERENCE, "include", "lotus", "vulkan_backend.hpp"))


def build_host(force=False, verbose=False):
    """Builds the adapter's test driver; returns its path, or None when the
    reference's headers are absent (a prebuilt driver is kept)."""
    if not reference_headers():
        return HARNESS if os.path.exists(HARNESS) else None
    sources = [os.path.join(HOST, "cuda_offscreen_renderer.cpp"),
               os.path.join(HERE, "..", "tests", "adapter_harness.cpp")]
    inputs = sources + [os.path.join(HOST, "cuda_offscreen_renderer.hpp"), LIB]
    if (not force and os.path.exists(HARNESS) and
            all(os.path.getmtime(p) <= os.path.getmtime(HARNESS) for p in inputs)):
        return HARNESS
    cmd = ["g++", "-std=c++20", "-O2", "-Wall", "-Wextra", f"-I{REFERENCE}/include"] + sources + \
          ["-o", HARNESS, f"-L{LIB_DIR}", "-llotus_cuda", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return HARNESS


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    build_table_tool(force="--force" in sys.argv, verbose=True)
    build_host(force="--force" in sys.argv, verbose=True)
