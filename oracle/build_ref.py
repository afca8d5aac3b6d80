"""Builds the reference's own CPU code for the temporal and reservoir paths
(TEST INFRASTRUCTURE ONLY).

Compiles, with g++ directly from the sources where they lie under the
reference tree ($LOTUS_REFERENCE, else ../reference beside this
checkout), into
oracle/_ref/:
  - libref.so: backend/vulkan/temporal.cpp, temporal_metadata.cpp,
    reservoir.cpp and core/render-world/render_world.cpp, with this
    directory's ref_bridge.cpp as a C interface;
  - the reference's own unit tests of that code, validation/
    reservoir-test.cpp, temporal-test.cpp and restir-statistics-test.cpp,
    whose passing run pins the build.
Where the reference tree is absent (as on a machine that only runs the
tests), the prebuilt files are used as they are.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("LOTUS_REFERENCE", os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
OUT = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT, "libref.so")
TESTS = ["reservoir-test", "temporal-test", "restir-statistics-test"]

SOURCES = ["backend/vulkan/temporal.cpp", "backend/vulkan/temporal_metadata.cpp",
           "backend/vulkan/reservoir.cpp", "core/render-world/render_world.cpp"]


def flags():
    return ["-std=c++20", "-O2", f"-I{REF}/include", f"-I{REF}/backend/vulkan", f"-I{REF}/validation"]


def available():
    return all(os.path.exists(os.path.join(REF, s)) for s in SOURCES)


def build(force=False, verbose=False):
    """Returns the library path, building it when the reference tree is
    present and the library is missing (or `force`)."""
    if not available():
        return LIB if os.path.exists(LIB) else None
    os.makedirs(OUT, exist_ok=True)
    srcs = [os.path.join(REF, s) for s in SOURCES]
    if force or not os.path.exists(LIB):
        cmd = ["g++", "-shared", "-fPIC"] + flags() + [os.path.join(HERE, "ref_bridge.cpp")] + srcs + ["-o", LIB]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    for t in TESTS:
        exe = os.path.join(OUT, t)
        if force or not os.path.exists(exe):
            cmd = ["g++"] + flags() + [os.path.join(REF, "validation", t + ".cpp")] + srcs + ["-o", exe]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
