"""ctypes wrapper of the oracle (TEST INFRASTRUCTURE ONLY).

The checker for the CUDA kernels: a scalar CPU restatement of the
reference's path tracer (oracle/lotus_oracle.cpp). Tests, the smoke check
and the benchmark's CPU-baseline leg use it; the product never does.
"""

import ctypes as C
import os

import numpy as np

from hydra_lotus_b200 import abi

from . import build as _build

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path):
            path = _build.build()
        L = C.CDLL(path)
        L.oracle_scene_create.restype = C.c_void_p
        L.oracle_scene_create.argtypes = [C.POINTER(abi.SceneDesc), C.c_char_p, C.c_size_t]
        L.oracle_scene_destroy.argtypes = [C.c_void_p]
        L.oracle_sample.restype = C.c_int32
        L.oracle_sample.argtypes = [C.c_void_p, C.POINTER(abi.FrameDesc), C.c_uint32,
                                    C.c_void_p, C.c_void_p, C.c_int32]
        L.oracle_accumulate.restype = C.c_int32
        L.oracle_accumulate.argtypes = [C.c_void_p, C.POINTER(abi.FrameDesc), C.c_uint32,
                                        C.c_uint32, C.c_void_p, C.c_void_p, C.c_int32]
        L.oracle_light_table.restype = C.c_int64
        L.oracle_light_table.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p,
                                         C.c_uint64]
        L.oracle_traversal_stats.restype = C.c_int32
        L.oracle_traversal_stats.argtypes = [C.c_void_p, C.POINTER(abi.FrameDesc), C.c_uint32,
                                             C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _lib = L
    return _lib


class OracleScene:
    def __init__(self, scene):
        self.scene = scene
        err = C.create_string_buffer(256)
        self.handle = lib().oracle_scene_create(C.byref(scene.desc()), err, 256)
        if not self.handle:
            raise RuntimeError("oracle scene: " + err.value.decode())

    def close(self):
        if self.handle:
            lib().oracle_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def sample(self, frame, sample_index, threads=0):
        """(H, W, 4) float32: each pixel's radiance and hit flag for one
        sample, and the (camera, extension, shadow) ray counts."""
        w, h = frame.target.width, frame.target.height
        out = np.zeros((h, w, 4), dtype=np.float32)
        rays = np.zeros(3, dtype=np.uint64)
        rc = lib().oracle_sample(self.handle, C.byref(frame), sample_index,
                                 out.ctypes.data, rays.ctypes.data, threads)
        if rc != abi.PASS:
            raise RuntimeError("oracle_sample failed")
        return out, rays

    def accumulate(self, frame, first_sample, count, sums=None, threads=0):
        """FP64 sums (H, W, 4) of `count` samples from `first_sample`."""
        w, h = frame.target.width, frame.target.height
        if sums is None:
            sums = np.zeros((h, w, 4), dtype=np.float64)
        rays = np.zeros(3, dtype=np.uint64)
        rc = lib().oracle_accumulate(self.handle, C.byref(frame), first_sample, count,
                                     sums.ctypes.data, rays.ctypes.data, threads)
        if rc != abi.PASS:
            raise RuntimeError("oracle_accumulate failed")
        return sums, rays

    def light_table(self):
        n = lib().oracle_light_table(self.handle, None, 0, None, 0)
        rec = np.zeros((max(n, 1), 4), dtype=np.uint32)
        off = np.zeros(max(1, len(self.scene.instances)), dtype=np.uint32)
        lib().oracle_light_table(self.handle, rec.ctypes.data, n, off.ctypes.data, off.size)
        return rec[:n], off[:len(self.scene.instances)]

    def traversal_stats(self, frame, max_rays=65536):
        nodes = C.c_double()
        tris = C.c_double()
        lib().oracle_traversal_stats(self.handle, C.byref(frame), max_rays, C.byref(nodes),
                                     C.byref(tris))
        return nodes.value, tris.value


def resolve(sums, clear_color=(0.0, 0.0, 0.0, 0.0), count=None):
    """The radiance pass's mean (path_trace.slang:369-384): a missed sample
    counts as the clear colour."""
    sums = np.asarray(sums, dtype=np.float64)
    if count is None:
        raise ValueError("count is required")
    bg = np.asarray(clear_color, dtype=np.float64)
    out = np.empty(sums.shape, dtype=np.float64)
    miss = count - sums[..., 3]
    out[..., :3] = (sums[..., :3] + miss[..., None] * bg[:3]) / count
    out[..., 3] = (sums[..., 3] + miss * bg[3]) / count
    return out
