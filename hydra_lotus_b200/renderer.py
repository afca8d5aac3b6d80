"""The Python host of the CUDA backend, mirroring the reference's
``Lotus::OffscreenRenderer`` (include/lotus/vulkan_backend.hpp:753-842 in
hydra-lotus) over the C ABI of include/lotus_cuda.h.

``CudaOffscreenRenderer.update_scene`` stands for ``UpdateScene``,
``render_scene`` for ``RenderScene``; both return the status and detail the
reference's evidence carries (Pass, Fail, Skip) instead of raising.
There is no CPU fallback: constructing a renderer without the compiled
library raises, and without an sm_100 device reports Skip.
"""

import ctypes as C
import os

import numpy as np

from . import abi
from . import build as _build

_lib = None


class LibraryMissing(RuntimeError):
    pass


def lib():
    """The loaded CUDA library. Raises LibraryMissing when it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(_build.LIB):
            raise LibraryMissing(
                f"{_build.LIB} is not built: run `python -m hydra_lotus_b200.build`")
        L = C.CDLL(_build.LIB)
        L.lotus_cuda_abi_version.restype = C.c_uint32
        L.lotus_cuda_struct_sizes.restype = C.c_uint32
        L.lotus_cuda_struct_sizes.argtypes = [C.POINTER(C.c_uint64), C.c_uint32]
        L.lotus_cuda_capability.restype = C.c_int32
        L.lotus_cuda_capability.argtypes = [C.c_int32, C.c_char_p, C.c_size_t]
        L.lotus_cuda_create.restype = C.c_int32
        L.lotus_cuda_create.argtypes = [C.POINTER(abi.Options), C.POINTER(C.c_void_p),
                                        C.c_char_p, C.c_size_t]
        L.lotus_cuda_destroy.argtypes = [C.c_void_p]
        L.lotus_cuda_update_scene.restype = C.c_int32
        L.lotus_cuda_update_scene.argtypes = [C.c_void_p, C.POINTER(abi.SceneDesc),
                                              C.POINTER(abi.SceneResult)]
        L.lotus_cuda_update_instances.restype = C.c_int32
        L.lotus_cuda_update_instances.argtypes = [C.c_void_p, C.POINTER(abi.Instance), C.c_uint32,
                                                  C.POINTER(abi.SceneResult)]
        L.lotus_cuda_update_geometry.restype = C.c_int32
        L.lotus_cuda_update_geometry.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(C.c_float), C.c_uint32,
                                                 C.POINTER(C.c_float), C.POINTER(abi.SceneResult)]
        L.lotus_cuda_render.restype = C.c_int32
        L.lotus_cuda_render.argtypes = [C.c_void_p, C.POINTER(abi.FrameDesc),
                                        C.POINTER(abi.FrameResult), C.c_void_p]
        L.lotus_cuda_read_color.restype = C.c_int32
        L.lotus_cuda_read_color.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64]
        L.lotus_cuda_read_depth.restype = C.c_int32
        L.lotus_cuda_read_depth.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64]
        L.lotus_cuda_read_scene.restype = C.c_int64
        L.lotus_cuda_read_scene.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint64]
        L.lotus_cuda_stream.restype = C.c_void_p
        L.lotus_cuda_stream.argtypes = [C.c_void_p]
        L.lotus_cuda_render_static.restype = C.c_int32
        L.lotus_cuda_render_static.argtypes = [C.c_void_p, C.POINTER(abi.FrameDesc), C.c_void_p,
                                               C.POINTER(abi.FrameResult)]
        L.lotus_cuda_set_temporal_instances.restype = C.c_int32
        L.lotus_cuda_set_temporal_instances.argtypes = [C.c_void_p, C.POINTER(abi.TemporalInstance),
                                                        C.c_uint32]
        L.lotus_cuda_render_temporal.restype = C.c_int32
        L.lotus_cuda_render_temporal.argtypes = [C.c_void_p, C.POINTER(abi.TemporalDesc),
                                                 C.POINTER(abi.FrameResult), C.c_void_p]
        L.lotus_cuda_read_product.restype = C.c_int64
        L.lotus_cuda_read_product.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64]
        L.lotus_cuda_configure_cache.restype = C.c_int32
        L.lotus_cuda_configure_cache.argtypes = [C.c_void_p, C.POINTER(abi.CacheDesc), C.c_char_p,
                                                 C.c_size_t]
        L.lotus_cuda_cache_weights.restype = C.c_int32
        L.lotus_cuda_cache_weights.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int32]
        L.lotus_cuda_cache_infer.restype = C.c_int32
        L.lotus_cuda_cache_infer.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
        L.lotus_cuda_cache_gradient.restype = C.c_int32
        L.lotus_cuda_cache_gradient.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                                C.c_void_p, C.c_void_p, C.c_void_p]
        L.lotus_cuda_cache_encode.restype = C.c_int32
        L.lotus_cuda_cache_encode.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
        L.lotus_cuda_cache_train.restype = C.c_int32
        L.lotus_cuda_cache_train.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                             C.c_void_p]
        L.lotus_cuda_batch_create.restype = C.c_int32
        L.lotus_cuda_batch_create.argtypes = [C.POINTER(abi.Options), C.POINTER(C.c_void_p), C.c_char_p,
                                              C.c_size_t]
        L.lotus_cuda_batch_destroy.restype = None
        L.lotus_cuda_batch_destroy.argtypes = [C.c_void_p]
        L.lotus_cuda_batch_set_scenes.restype = C.c_int32
        L.lotus_cuda_batch_set_scenes.argtypes = [C.c_void_p, C.POINTER(abi.SceneDesc), C.c_uint32,
                                                  C.POINTER(abi.SceneResult)]
        L.lotus_cuda_batch_set_tuning.restype = C.c_int32
        L.lotus_cuda_batch_set_tuning.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]
        L.lotus_cuda_batch_render.restype = C.c_int32
        L.lotus_cuda_batch_render.argtypes = [C.c_void_p, C.POINTER(abi.FrameDesc), C.c_uint32,
                                              C.POINTER(abi.FrameResult), C.POINTER(C.c_void_p),
                                              C.POINTER(abi.FrameResult)]
        L.lotus_cuda_read_light_table.restype = C.c_int64
        L.lotus_cuda_read_light_table.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64,
                                                  C.c_void_p, C.c_uint64]
        if L.lotus_cuda_abi_version() != abi.ABI_VERSION:
            raise RuntimeError("liblotus_cuda ABI version mismatch")
        abi.check_struct_sizes(L)
        _lib = L
    return _lib


def capability(device=0):
    """RayQueryCapability: (status, detail)."""
    buf = C.create_string_buffer(256)
    status = lib().lotus_cuda_capability(device, buf, 256)
    return status, buf.value.decode()


class RendererError(RuntimeError):
    def __init__(self, status, detail):
        super().__init__(f"status {status}: {detail}")
        self.status = status
        self.detail = detail


class CudaOffscreenRenderer:
    """One renderer: one device, one stream, the resident scene and the
    accumulation targets."""

    def __init__(self, device=0, bvh_leaf_size=0, trace_refill_below=0, trace_blocks_per_sm=0,
                 wavefront_rounds=0, traversal_step_limit=0, samples_per_wave=0):
        self.handle = None
        opts = abi.Options(device=device, flags=0, bvh_leaf_size=bvh_leaf_size,
                           trace_refill_below=trace_refill_below, trace_blocks_per_sm=trace_blocks_per_sm,
                           wavefront_rounds=wavefront_rounds, traversal_step_limit=traversal_step_limit,
                           samples_per_wave=samples_per_wave)
        h = C.c_void_p()
        err = C.create_string_buffer(256)
        status = lib().lotus_cuda_create(C.byref(opts), C.byref(h), err, 256)
        if status != abi.PASS:
            raise RendererError(status, err.value.decode())
        self.handle = h
        self.scene = None

    def close(self):
        if self.handle:
            lib().lotus_cuda_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def stream(self):
        """The renderer's cudaStream_t as an integer handle."""
        return lib().lotus_cuda_stream(self.handle)

    def update_scene(self, scene):
        """UpdateScene: uploads `scene` (a scenes.Scene). Returns the
        lotus_scene_result."""
        res = abi.SceneResult()
        lib().lotus_cuda_update_scene(self.handle, C.byref(scene.desc()), C.byref(res))
        self.scene = scene
        return res

    def update_instances(self, scene):
        """UpdateScene for an instance-only change (lotus_cuda_update_instances):
        the resident scene takes `scene`'s instances; its geometries,
        materials and environment stay as uploaded. Returns the
        lotus_scene_result."""
        d = scene.desc()
        res = abi.SceneResult()
        lib().lotus_cuda_update_instances(self.handle, d.instances, d.instance_count, C.byref(res))
        self.scene = scene
        return res

    def update_geometry(self, scene, geometry):
        """UpdateScene for a point edit (lotus_cuda_update_geometry): the
        resident geometry `geometry` takes `scene`'s positions (and corner
        normals) for it. Returns the lotus_scene_result."""
        p, _, n = scene.geometries[geometry]
        res = abi.SceneResult()
        lib().lotus_cuda_update_geometry(
            self.handle, geometry, p.ctypes.data_as(C.POINTER(C.c_float)), p.shape[0],
            n.ctypes.data_as(C.POINTER(C.c_float)) if n is not None else C.POINTER(C.c_float)(), C.byref(res))
        self.scene = scene
        return res

    def render_scene(self, frame, color=None):
        """RenderScene: returns (lotus_frame_result, colour). With
        frame.target.read_back, colour is an (H, W, 4) float32 array (or the
        given one, filled)."""
        res = abi.FrameResult()
        ptr = None
        if frame.target.read_back:
            if color is None:
                color = np.empty((frame.target.height, frame.target.width, 4), dtype=np.float32)
            ptr = color.ctypes.data
        lib().lotus_cuda_render(self.handle, C.byref(frame), C.byref(res), ptr)
        return res, (color if frame.target.read_back else None)

    def render_static(self, frame, color_device_ptr):
        """lotus_cuda_render_static: renders `frame` into caller-owned device
        memory (an integer device pointer to width*height*4 floats) without
        allocating. Returns the lotus_frame_result."""
        res = abi.FrameResult()
        lib().lotus_cuda_render_static(self.handle, C.byref(frame), C.c_void_p(color_device_ptr),
                                       C.byref(res))
        return res

    def render_temporal(self, temporal, color=None):
        """RenderTemporalScene: returns (lotus_frame_result, colour)."""
        res = abi.FrameResult()
        t = temporal.frame.target
        ptr = None
        if t.read_back:
            if color is None:
                color = np.empty((t.height, t.width, 4), dtype=np.float32)
            ptr = color.ctypes.data
        lib().lotus_cuda_render_temporal(self.handle, C.byref(temporal), C.byref(res), ptr)
        return res, (color if t.read_back else None)

    def set_temporal_instances(self, records):
        arr = (abi.TemporalInstance * max(1, len(records)))(*records)
        rc = lib().lotus_cuda_set_temporal_instances(self.handle, arr, len(records))
        if rc != abi.PASS:
            raise RendererError(rc, "set_temporal_instances failed")

    def read_product(self, product, height, width):
        """A temporal product as a structured (H, W) numpy array."""
        dtype = abi.PRODUCT_DTYPES[product]
        out = np.zeros((height, width), dtype=dtype)
        n = lib().lotus_cuda_read_product(self.handle, product, out.ctypes.data, out.nbytes)
        if n < 0:
            raise RendererError(abi.FAIL, f"product {product} is not available")
        return out

    def read_scene(self, what, index=0):
        """ReadBackScene: a copy of the resident scene as the device holds
        it (abi.SCENE_*): positions (n, 3), triangles (n, 3), corner normals
        (n, 3, 3) of geometry `index`; every instance or material as ctypes
        records; the constant environment (3,)."""
        n = lib().lotus_cuda_read_scene(self.handle, what, index, None, 0)
        if n < 0:
            raise RendererError(abi.FAIL, f"scene readback {what} failed")
        buf = (C.c_uint8 * max(int(n), 1))()
        if lib().lotus_cuda_read_scene(self.handle, what, index, C.addressof(buf), n) != n:
            raise RendererError(abi.FAIL, f"scene readback {what} failed")
        raw = bytes(buf)[:n]
        if what == abi.SCENE_POSITIONS:
            return np.frombuffer(raw, np.float32).reshape(-1, 3)
        if what == abi.SCENE_TRIANGLES:
            return np.frombuffer(raw, np.uint32).reshape(-1, 3)
        if what == abi.SCENE_NORMALS:
            return np.frombuffer(raw, np.float32).reshape(-1, 3, 3)
        if what == abi.SCENE_ENVIRONMENT:
            return np.frombuffer(raw, np.float32)
        rec = abi.Instance if what == abi.SCENE_INSTANCES else abi.Material
        count = n // C.sizeof(rec)
        return list((rec * count).from_buffer_copy(raw)) if count else []

    def read_depth(self, height, width):
        """The latest frame's depth product (LOTUS_FRAME_DEPTH): (H, W)
        float32 Vulkan window depth, top-left rows."""
        out = np.empty((height, width), dtype=np.float32)
        rc = lib().lotus_cuda_read_depth(self.handle, out.ctypes.data, out.size)
        if rc != abi.PASS:
            raise RendererError(rc, "read_depth failed: no depth product")
        return out

    def read_color(self, out):
        rc = lib().lotus_cuda_read_color(self.handle, out.ctypes.data, out.size)
        if rc != abi.PASS:
            raise RendererError(rc, "read_color failed")
        return out

    # --- the learned radiance cache -------------------------------------

    def configure_cache(self, enable=True, **fields):
        """lotus_cuda_configure_cache: fresh weights over the resident
        scene's bounds; `fields` are lotus_cache_desc members."""
        d = abi.CacheDesc(enable=1 if enable else 0, **fields)
        err = C.create_string_buffer(256)
        rc = lib().lotus_cuda_configure_cache(self.handle, C.byref(d), err, 256)
        if rc != abi.PASS:
            raise RendererError(rc, err.value.decode(errors="replace"))

    def cache_weights(self, weights=None):
        """Reads the cache's FP32 weights, or writes `weights`."""
        if weights is None:
            w = np.zeros(abi.CACHE_WEIGHTS, dtype=np.float32)
            rc = lib().lotus_cuda_cache_weights(self.handle, w.ctypes.data, w.size, 0)
        else:
            w = np.ascontiguousarray(weights, dtype=np.float32).ravel()
            rc = lib().lotus_cuda_cache_weights(self.handle, w.ctypes.data, w.size, 1)
        if rc != abi.PASS:
            raise RendererError(rc, "cache weights")
        return w

    def cache_infer(self, inputs):
        x = np.ascontiguousarray(inputs, dtype=np.float32)
        out = np.zeros((x.shape[0], 3), dtype=np.float32)
        rc = lib().lotus_cuda_cache_infer(self.handle, x.ctypes.data, x.shape[0], out.ctypes.data)
        if rc != abi.PASS:
            raise RendererError(rc, "cache inference")
        return out

    def cache_gradient(self, inputs, targets):
        """(weight gradients, input gradients, loss) of the relative L2 loss."""
        x = np.ascontiguousarray(inputs, dtype=np.float32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        gw = np.zeros(abi.CACHE_WEIGHTS, dtype=np.float32)
        gx = np.zeros_like(x)
        loss = np.zeros(1, dtype=np.float32)
        rc = lib().lotus_cuda_cache_gradient(self.handle, x.ctypes.data, t.ctypes.data, x.shape[0],
                                             gw.ctypes.data, gx.ctypes.data, loss.ctypes.data)
        if rc != abi.PASS:
            raise RendererError(rc, "cache gradient")
        return gw, gx, float(loss[0])

    def cache_encode(self, records):
        r = np.ascontiguousarray(records, dtype=np.float32)
        out = np.zeros((r.shape[0], abi.CACHE_INPUTS), dtype=np.float32)
        rc = lib().lotus_cuda_cache_encode(self.handle, r.ctypes.data, r.shape[0], out.ctypes.data)
        if rc != abi.PASS:
            raise RendererError(rc, "cache encode")
        return out

    def cache_train(self, records, targets, steps):
        """Trains on raw records; returns the loss before each step."""
        r = np.ascontiguousarray(records, dtype=np.float32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        losses = np.zeros(steps, dtype=np.float32)
        rc = lib().lotus_cuda_cache_train(self.handle, r.ctypes.data, t.ctypes.data, r.shape[0], steps,
                                          losses.ctypes.data)
        if rc != abi.PASS:
            raise RendererError(rc, "cache training")
        return losses

    def light_table(self):
        n = lib().lotus_cuda_read_light_table(self.handle, None, 0, None, 0)
        if n < 0:
            raise RendererError(abi.FAIL, "no light table")
        ninst = len(self.scene.instances) if self.scene else 0
        rec = np.zeros((max(n, 1), 4), dtype=np.uint32)
        off = np.zeros(max(ninst, 1), dtype=np.uint32)
        lib().lotus_cuda_read_light_table(self.handle, rec.ctypes.data, n, off.ctypes.data, ninst)
        return rec[:n], off[:ninst]


class CudaBatch:
    """Several scenes rendered as one wavefront (lotus_cuda_batch_*)."""

    def __init__(self, device=0, trace_refill_below=0, trace_blocks_per_sm=0, wavefront_rounds=0):
        self.handle = None
        opts = abi.Options(device=device, flags=0, trace_refill_below=trace_refill_below,
                           trace_blocks_per_sm=trace_blocks_per_sm, wavefront_rounds=wavefront_rounds)
        h = C.c_void_p()
        err = C.create_string_buffer(256)
        status = lib().lotus_cuda_batch_create(C.byref(opts), C.byref(h), err, 256)
        if status != abi.PASS:
            raise RendererError(status, err.value.decode(errors="replace"))
        self.handle = h
        self.scenes = []

    def close(self):
        if self.handle:
            lib().lotus_cuda_batch_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_scenes(self, scenes):
        """Builds every scene; returns their lotus_scene_result."""
        self.scenes = list(scenes)
        descs = (abi.SceneDesc * len(self.scenes))(*[s.desc() for s in self.scenes])
        results = (abi.SceneResult * len(self.scenes))()
        lib().lotus_cuda_batch_set_scenes(self.handle, descs, len(self.scenes), results)
        return list(results)

    def set_tuning(self, refill_below=0, blocks_per_sm=0, wavefront_rounds=0, camera_tile=0):
        """The batch's launch shape (lotus_cuda_batch_set_tuning; 0: each
        default); camera_tile is one of abi.CAMERA_TILE_*."""
        rc = lib().lotus_cuda_batch_set_tuning(self.handle, refill_below, blocks_per_sm, wavefront_rounds,
                                               camera_tile)
        if rc != abi.PASS:
            raise RendererError(rc, "batch tuning")

    def render(self, frames):
        """frames[k] renders scene k: (per-scene results, per-scene colours
        (H, W, 4) or None, the call's total)."""
        n = len(frames)
        fa = (abi.FrameDesc * n)(*frames)
        results = (abi.FrameResult * n)()
        colors, ptrs = [], (C.c_void_p * n)()
        for k, f in enumerate(frames):
            if f.target.read_back:
                c = np.empty((f.target.height, f.target.width, 4), dtype=np.float32)
                colors.append(c)
                ptrs[k] = c.ctypes.data
            else:
                colors.append(None)
        total = abi.FrameResult()
        lib().lotus_cuda_batch_render(self.handle, fa, n, results, ptrs, C.byref(total))
        return list(results), colors, total


def check(result, what="call"):
    """Raises RendererError unless `result.status` is Pass."""
    if result.status != abi.PASS:
        raise RendererError(result.status, f"{what}: {result.detail.decode(errors='replace')}")
    return result
