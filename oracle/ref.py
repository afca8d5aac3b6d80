"""ctypes wrapper of the reference's own CPU temporal and reservoir code
(TEST INFRASTRUCTURE ONLY), built by oracle/build_ref.py into oracle/_ref/.

The checker for the SVGF, reprojection and reservoir kernels; the product
never loads it.
"""

import ctypes as C
import os

import numpy as np

from . import build_ref

_lib = None


def available():
    return build_ref.build() is not None and os.path.exists(build_ref.LIB)


def lib():
    global _lib
    if _lib is None:
        path = build_ref.build()
        if path is None or not os.path.exists(path):
            raise RuntimeError("oracle/_ref/libref.so is not built (needs the reference tree once)")
        L = C.CDLL(path)
        vp = C.c_void_p
        L.ref_estimate_variance.restype = C.c_float
        L.ref_estimate_variance.argtypes = [vp, vp] + [C.c_uint32] * 6
        L.ref_filter.restype = C.c_int
        L.ref_filter.argtypes = [vp, vp] + [C.c_uint32] * 5 + [vp]
        L.ref_reproject.restype = None
        L.ref_reproject.argtypes = [vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, vp, C.c_uint64, vp, vp]
        L.ref_stream_candidate.restype = C.c_int
        L.ref_stream_candidate.argtypes = [vp, C.c_uint32, C.c_float, C.c_float, C.c_float, C.POINTER(C.c_int)]
        L.ref_merge_reevaluated.restype = C.c_int
        L.ref_merge_reevaluated.argtypes = [vp, vp, C.c_double, C.c_float, C.c_uint32, C.c_float,
                                            C.POINTER(C.c_int)]
        L.ref_normalization.restype = C.c_double
        L.ref_normalization.argtypes = [vp, C.POINTER(C.c_int)]
        L.ref_reuse_normalization.restype = C.c_double
        L.ref_reuse_normalization.argtypes = [vp, C.c_uint32, C.POINTER(C.c_int)]
        _lib = L
    return _lib


def estimate_variance(surface, radiance, batch_samples, max_history):
    """EstimateTemporalVariance at every pixel: (H, W) float32."""
    h, w = surface.shape
    out = np.zeros((h, w), dtype=np.float32)
    L = lib()
    for y in range(h):
        for x in range(w):
            out[y, x] = L.ref_estimate_variance(surface.ctypes.data, radiance.ctypes.data, x, y, w, h,
                                                batch_samples, max_history)
    return out


def filter_composite(surface, radiance, batch_samples, max_history, iterations):
    """FilterTemporalRadiance: (H, W, 4) float32 composite."""
    h, w = surface.shape
    out = np.zeros((h, w, 4), dtype=np.float32)
    rc = lib().ref_filter(surface.ctypes.data, radiance.ctypes.data, w, h, batch_samples, max_history,
                          iterations, out.ctypes.data)
    if rc != 0:
        raise RuntimeError("FilterTemporalRadiance rejected its input")
    return out


def reproject(current, previous, validation):
    """ReprojectTemporalHistory at every pixel, with `previous` the
    preceding frame's records (or an empty array after a reset)."""
    from hydra_lotus_b200 import abi
    h, w = current.shape
    out = np.zeros((h, w), dtype=abi.VALIDITY_PIXEL)
    v = np.asarray(validation, dtype=np.float32)
    L = lib()
    prev = np.ascontiguousarray(previous)
    n = prev.size
    for y in range(h):
        for x in range(w):
            L.ref_reproject(current[y, x:x + 1].ctypes.data, x, y, w, h, prev.ctypes.data if n else None, n,
                            v.ctypes.data, out[y, x:x + 1].ctypes.data)
    return out
