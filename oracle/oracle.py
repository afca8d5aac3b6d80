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


class OracleTemporal(C.Structure):
    """oracle_temporal: the temporal passes' constants."""
    _fields_ = [
        ("current_view", C.c_float * 16),
        ("previous_view", C.c_float * 16),
        ("previous_world_to_clip", C.c_float * 16),
        ("previous_display", C.c_float * 4),
        ("previous_data", C.c_uint32 * 4),
        ("restir_candidates", C.c_uint32),
        ("restir_history", C.c_uint32),
        ("restir_max_history", C.c_uint32),
        ("restir_radius", C.c_uint32),
        ("restir_neighbours", C.c_uint32),
        ("restir_proposal", C.c_uint32),
        ("max_bounces", C.c_uint32),
    ]


def vulkan_clip(world_to_clip):
    """VulkanWorldToClip (vulkan_internal.hpp:326-336) in float32."""
    m = np.asarray(world_to_clip, dtype=np.float32).copy()
    for c in range(4):
        y, z, w = m[c * 4 + 1], m[c * 4 + 2], m[c * 4 + 3]
        m[c * 4 + 1] = -y
        m[c * 4 + 2] = np.float32(0.5) * np.float32(z + w)
    return m


def oracle_temporal(temporal_desc):
    """The oracle's constants for a lotus_temporal_desc, as the renderer
    derives them (whole-image display and data windows)."""
    f = temporal_desc.frame
    st = f.settings
    t = OracleTemporal()
    t.current_view[:] = list(temporal_desc.current_view)
    if temporal_desc.history_available:
        t.previous_view[:] = list(temporal_desc.previous_view)
        t.previous_world_to_clip[:] = [float(v) for v in vulkan_clip(temporal_desc.previous_world_to_clip)]
    t.previous_display[:] = [0.0, 0.0, float(f.target.width), float(f.target.height)]
    t.previous_data[:] = [0, 0, f.target.width, f.target.height]
    t.restir_candidates = st.restir_candidates
    t.restir_history = 1 if (st.restir_temporal and temporal_desc.history_available) else 0
    t.restir_max_history = st.restir_max_history_candidates
    t.restir_radius = st.restir_spatial_radius
    t.restir_neighbours = st.restir_spatial_neighbours
    t.restir_proposal = st.restir_proposal
    t.max_bounces = st.max_bounces
    return t


def _temporal_lib():
    L = lib()
    if not hasattr(L, "_temporal_ready"):
        vp = C.c_void_p
        L.oracle_temporal_surface.restype = C.c_int32
        L.oracle_temporal_surface.argtypes = [vp, C.POINTER(abi.FrameDesc), C.POINTER(OracleTemporal), vp, vp]
        L.oracle_restir_initial.restype = C.c_int32
        L.oracle_restir_initial.argtypes = [vp, C.POINTER(abi.FrameDesc), C.POINTER(OracleTemporal),
                                            C.c_uint32, vp]
        L.oracle_restir_temporal.restype = C.c_int32
        L.oracle_restir_temporal.argtypes = [vp, C.POINTER(abi.FrameDesc), C.POINTER(OracleTemporal), vp,
                                             C.c_uint32, vp, vp, vp, vp, vp, vp, vp]
        L.oracle_restir_spatial.restype = C.c_int32
        L.oracle_restir_spatial.argtypes = [vp, C.POINTER(abi.FrameDesc), C.POINTER(OracleTemporal),
                                            C.c_uint32, vp, vp, vp, vp]
        L.oracle_sample_restir.restype = C.c_int32
        L.oracle_sample_restir.argtypes = [vp, C.POINTER(abi.FrameDesc), C.c_uint32, vp, C.c_uint32, vp, vp,
                                           C.c_int32]
        L._temporal_ready = True
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data


class OracleTemporalScene(OracleScene):
    """The oracle's temporal passes over the kernels' record layouts."""

    def temporal_surface(self, frame, tc, ids=None):
        h, w = frame.target.height, frame.target.width
        out = np.zeros((h, w), dtype=abi.TEMPORAL_PIXEL)
        ids_arr = None if ids is None else (abi.TemporalInstance * len(ids))(*ids)
        _temporal_lib().oracle_temporal_surface(self.handle, C.byref(frame), C.byref(tc),
                                                C.cast(ids_arr, C.c_void_p) if ids_arr else None,
                                                out.ctypes.data)
        return out

    def restir_initial(self, frame, tc, sample_index):
        h, w = frame.target.height, frame.target.width
        out = np.zeros((h, w), dtype=abi.RESTIR_PIXEL)
        _temporal_lib().oracle_restir_initial(self.handle, C.byref(frame), C.byref(tc), sample_index,
                                              out.ctypes.data)
        return out

    def restir_temporal(self, frame, tc, sample_index, initial, validity, surface, previous,
                        previous_surfaces, ids=None):
        h, w = frame.target.height, frame.target.width
        out = np.zeros((h, w), dtype=abi.RESTIR_REUSE)
        out_s = np.zeros((h, w), dtype=abi.RESTIR_SURFACE)
        ids_arr = None if ids is None else (abi.TemporalInstance * len(ids))(*ids)
        _temporal_lib().oracle_restir_temporal(
            self.handle, C.byref(frame), C.byref(tc), C.cast(ids_arr, C.c_void_p) if ids_arr else None,
            sample_index, _ptr(initial), _ptr(validity), _ptr(surface), _ptr(previous),
            _ptr(previous_surfaces), out.ctypes.data, out_s.ctypes.data)
        return out, out_s

    def restir_spatial(self, frame, tc, sample_index, temporal, surfaces):
        h, w = frame.target.height, frame.target.width
        out = np.zeros((h, w), dtype=abi.RESTIR_REUSE)
        src = np.zeros((h, w, 4), dtype=np.uint32)
        _temporal_lib().oracle_restir_spatial(self.handle, C.byref(frame), C.byref(tc), sample_index,
                                              _ptr(temporal), _ptr(surfaces), out.ctypes.data,
                                              src.ctypes.data)
        return out, src

    def sample_restir(self, frame, sample_index, final_records, threads=0):
        h, w = frame.target.height, frame.target.width
        out = np.zeros((h, w, 4), dtype=np.float32)
        rays = np.zeros(3, dtype=np.uint64)
        rc = _temporal_lib().oracle_sample_restir(self.handle, C.byref(frame), sample_index,
                                                  final_records.ctypes.data, final_records.dtype.itemsize,
                                                  out.ctypes.data, rays.ctypes.data, threads)
        if rc != abi.PASS:
            raise RuntimeError("oracle_sample_restir failed")
        return out, rays
