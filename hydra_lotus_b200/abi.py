"""ctypes mirrors of the plain-data structs in include/lotus_cuda.h.

The C ABI is the boundary that replaces the reference's
``Lotus::OffscreenRenderer`` (include/lotus/vulkan_backend.hpp:753-842 in
hydra-lotus); these mirrors let Python hosts, tests and the benchmark fill
and read its structs. ``check_struct_sizes`` compares them with the sizes
the compiled library reports.
"""

import ctypes as C

PASS = 0
FAIL = 1
SKIP = 77

INTEGRATOR_REFERENCE = 0
INTEGRATOR_WAVEFRONT = 1

LIGHT_SAMPLING_BSDF = 0
LIGHT_SAMPLING_MIS = 1
LIGHT_SAMPLING_RESTIR_INITIAL = 2

MAX_BOUNCES = 1024
MAX_REPORTED_BOUNCES = 64
WAVEFRONT_ROUNDS = 9

STATIC_MAX_PIXELS = 65536

FRAME_TIMINGS = 1
FRAME_COUNT_VISITS = 2
FRAME_DEPTH = 4

SCENE_POSITIONS = 1
SCENE_TRIANGLES = 2
SCENE_NORMALS = 3
SCENE_INSTANCES = 4
SCENE_MATERIALS = 5
SCENE_ENVIRONMENT = 6
FRAME_DEPTH_KEEP = 8

# lotus_cuda_batch_set_tuning's camera order.
CAMERA_TILE_ROWS = 1
CAMERA_TILE_4X8 = 2
CAMERA_TILE_8X4 = 3
CAMERA_TILE_16X2 = 4

MOMENTS_FP32 = 0
MOMENTS_FP16 = 1

# Texture lookups (lotus_texture, lotus_texture_input, lotus_material::lookups).
TEXTURE_RGBA8_UNORM = 0
TEXTURE_RGBA8_SRGB = 1
TEXTURE_RGBA32_FLOAT = 2
WRAP_BLACK = 0
WRAP_CLAMP = 1
WRAP_REPEAT = 2
WRAP_MIRROR = 3
SLOT_OPACITY = 0
SLOT_NORMAL = 1
SLOT_BASE_COLOR = 2
SLOT_ROUGHNESS = 3
SLOT_METALLIC = 4
SLOT_EMISSION = 5
SLOT_SPECULAR_COLOR = 6
# glTF PBR's slots (0 and 1 are the geometry's, as above).
GLTF_SLOT_BASE_COLOR = 2
GLTF_SLOT_METALLIC = 3
GLTF_SLOT_ROUGHNESS = 4
GLTF_SLOT_EMISSIVE = 5
GLTF_SLOT_SPECULAR = 6
GLTF_SLOT_SPECULAR_COLOR = 7
GLTF_SLOT_TRANSMISSION = 8
GLTF_SLOT_CLEARCOAT = 9
GLTF_SLOT_CLEARCOAT_ROUGHNESS = 10
GLTF_SLOT_CLEARCOAT_NORMAL = 11
GLTF_SLOT_SHEEN_COLOR = 12
GLTF_SLOT_SHEEN_ROUGHNESS = 13
TEXTURE_SLOTS = 14

MATERIAL_SPECULAR_WORKFLOW = 1
MATERIAL_THIN_WALLED = 2
# lotus_material::model (ShadingModel).
MODEL_PREVIEW_SURFACE = 0
MODEL_GLTF_PBR = 1

ABI_VERSION = 10

# lotus_settings::output (SceneOutput).
OUTPUT_RADIANCE = 0
OUTPUT_BARYCENTRICS = 1
OUTPUT_SHADING_NORMAL = 2
OUTPUT_ALBEDO = 3
OUTPUT_ROUGHNESS_METALLIC = 4


class Geometry(C.Structure):
    _fields_ = [
        ("positions", C.POINTER(C.c_float)),
        ("triangles", C.POINTER(C.c_uint32)),
        ("normals", C.POINTER(C.c_float)),
        ("vertex_count", C.c_uint32),
        ("triangle_count", C.c_uint32),
        ("texcoords", C.POINTER(C.c_float)),
        ("texcoord_sets", C.c_uint32),
        ("color_sets", C.c_uint32),
        ("colors", C.POINTER(C.c_float)),
        ("color_counts", C.POINTER(C.c_uint32)),
    ]


class Instance(C.Structure):
    _fields_ = [
        ("world_from_object", C.c_float * 16),
        ("geometry", C.c_uint32),
        ("material", C.c_uint32),
        ("texcoord_set", C.c_uint32),  # k > 0: the geometry's set k - 1; 0: none
        ("color_set", C.c_uint32),  # k > 0: the geometry's colour set k - 1; 0: none
    ]


class Texture(C.Structure):
    _fields_ = [
        ("texels", C.c_void_p),
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("format", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


class TextureInput(C.Structure):
    _fields_ = [
        ("texture", C.c_uint32),  # k > 0: textures[k - 1]; 0: none (the fallback)
        ("channel", C.c_uint32),
        ("wrap_s", C.c_uint32),
        ("wrap_t", C.c_uint32),
        ("scale", C.c_float * 4),
        ("bias", C.c_float * 4),
        ("fallback", C.c_float * 4),
        ("st_transform", C.c_float * 6),
        ("reserved", C.c_uint32 * 2),
    ]


class Material(C.Structure):
    _fields_ = [
        ("base_color", C.c_float * 3),
        ("roughness", C.c_float),
        ("emission", C.c_float * 3),
        ("metallic", C.c_float),
        ("specular_color", C.c_float * 3),
        ("ior", C.c_float),
        ("transmission_color", C.c_float * 3),
        ("transmission", C.c_float),
        ("opacity", C.c_float),
        ("opacity_threshold", C.c_float),
        ("flags", C.c_uint32),
        ("model", C.c_uint32),  # MODEL_*
        ("lookups", C.c_uint32 * 14),  # per slot: k > 0 for texture_inputs[k - 1]; 0: the constant
        ("texcoord_fallback", C.c_float * 2),
        ("normal", C.c_float * 3),  # tangent-space shading normal; all zero: (0, 0, 1)
        # glTF PBR's inputs beyond the shared fields above.
        ("emissive_strength", C.c_float),
        ("specular", C.c_float),
        ("clearcoat", C.c_float),
        ("clearcoat_roughness", C.c_float),
        ("sheen_color", C.c_float * 3),
        ("sheen_roughness", C.c_float),
    ]


class Environment(C.Structure):
    _fields_ = [
        ("texels", C.POINTER(C.c_float)),
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("scale", C.c_float * 3),
        ("environment_from_world", C.c_float * 9),
    ]


# lotus_light::shape (LightShape).
LIGHT_SPHERE = 0
LIGHT_RECT = 1
LIGHT_DISK = 2
LIGHT_DISTANT = 3


class Light(C.Structure):
    _fields_ = [
        ("shape", C.c_uint32),
        ("normalize", C.c_uint32),
        ("world_from_light", C.c_float * 16),
        ("radiance", C.c_float * 3),
        ("radius", C.c_float),
        ("width", C.c_float),
        ("height", C.c_float),
        ("angle", C.c_float),
        ("reserved", C.c_uint32),
    ]


class SceneDesc(C.Structure):
    _fields_ = [
        ("geometries", C.POINTER(Geometry)),
        ("instances", C.POINTER(Instance)),
        ("materials", C.POINTER(Material)),
        ("environment", C.POINTER(Environment)),
        ("geometry_count", C.c_uint32),
        ("instance_count", C.c_uint32),
        ("material_count", C.c_uint32),
        ("environment_constant", C.c_float * 3),
        ("lights", C.POINTER(Light)),
        ("light_count", C.c_uint32),
        ("textures", C.POINTER(Texture)),
        ("texture_count", C.c_uint32),
        ("texture_input_count", C.c_uint32),
        ("texture_inputs", C.POINTER(TextureInput)),
    ]


class SceneResult(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("triangle_count", C.c_uint32),
        ("instance_count", C.c_uint32),
        ("light_count", C.c_uint32),
        ("bvh_node_count", C.c_uint32),
        ("tlas_node_count", C.c_uint32),
        ("build_gpu_ms", C.c_double),
        ("device_bytes", C.c_uint64),
        ("detail", C.c_char * 256),
    ]


class Target(C.Structure):
    _fields_ = [
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("display_window", C.c_float * 4),
        ("data_window", C.c_int32 * 4),
        ("clear_color", C.c_float * 4),
        ("read_back", C.c_uint32),
        ("clear_depth", C.c_float),
    ]


class Settings(C.Structure):
    _fields_ = [
        ("integrator", C.c_uint32),
        ("light_sampling", C.c_uint32),
        ("sample_index", C.c_uint32),
        ("max_bounces", C.c_uint32),
        ("max_samples", C.c_uint32),
        ("restir_candidates", C.c_uint32),
        ("restir_temporal", C.c_uint32),
        ("restir_max_history_candidates", C.c_uint32),
        ("restir_spatial", C.c_uint32),
        ("restir_spatial_radius", C.c_uint32),
        ("restir_proposal", C.c_uint32),
        ("environment_background", C.c_uint32),
        ("output", C.c_uint32),
        ("restir_spatial_neighbours", C.c_uint32),
    ]


class FrameDesc(C.Structure):
    _fields_ = [
        ("world_to_clip", C.c_float * 16),
        ("target", Target),
        ("settings", Settings),
        ("frame_count", C.c_uint32),
        ("flags", C.c_uint32),
    ]


class FrameResult(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("frames_rendered", C.c_uint32),
        ("samples_per_pixel", C.c_uint32),
        ("wavefront_rounds", C.c_uint32),
        ("completion", C.c_uint64),
        ("camera_rays", C.c_uint64),
        ("extension_rays", C.c_uint64),
        ("shadow_rays", C.c_uint64),
        ("gpu_ms", C.c_double),
        ("wavefront_path_counts", C.c_uint32 * MAX_REPORTED_BOUNCES),
        ("wavefront_path_count_size", C.c_uint32),
        ("timings_available", C.c_uint32),
        ("camera_gpu_ms", C.c_double),
        ("extend_gpu_ms", C.c_double),
        ("shade_gpu_ms", C.c_double),
        ("shadow_gpu_ms", C.c_double),
        ("resolve_gpu_ms", C.c_double),
        ("extend_launches", C.c_uint32),
        ("shadow_launches", C.c_uint32),
        ("visit_rays", C.c_uint64 * 3),
        ("node_visits", C.c_uint64 * 3),
        ("triangle_visits", C.c_uint64 * 3),
        ("instance_visits", C.c_uint64 * 3),
        ("cache_gpu_ms", C.c_double),
        ("cache_queries", C.c_uint32),
        ("cache_training_records", C.c_uint32),
        ("tail_gpu_ms", C.c_double),
        ("last_wave_samples", C.c_uint32),
        ("reserved", C.c_uint32),
        ("sort_gpu_ms", C.c_double),
        ("cache_infer_gpu_ms", C.c_double),
        ("cache_train_gpu_ms", C.c_double),
        ("detail", C.c_char * 256),
    ]


class Options(C.Structure):
    _fields_ = [("device", C.c_int32), ("flags", C.c_uint32), ("bvh_leaf_size", C.c_uint32),
                ("trace_refill_below", C.c_uint32), ("trace_blocks_per_sm", C.c_uint32),
                ("wavefront_rounds", C.c_uint32), ("traversal_step_limit", C.c_uint32),
                ("samples_per_wave", C.c_uint32)]


class TemporalDesc(C.Structure):
    _fields_ = [
        ("frame", FrameDesc),
        ("current_view", C.c_float * 16),
        ("previous_view", C.c_float * 16),
        ("previous_world_to_clip", C.c_float * 16),
        ("validation", C.c_float * 4),
        ("history_available", C.c_uint32),
        ("accumulate_radiance", C.c_uint32),
        ("max_history_samples", C.c_uint32),
        ("filter_iterations", C.c_uint32),
        ("history_rectification", C.c_uint32),
        ("moment_precision", C.c_uint32),
    ]


class TemporalInstance(C.Structure):
    _fields_ = [
        ("previous_world_from_object", C.c_float * 16),
        ("instance_id", C.c_uint64),
        ("material_id", C.c_uint64),
        ("flags", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


# The order lotus_cuda_struct_sizes reports them in.
class CacheDesc(C.Structure):
    """lotus_cache_desc: the learned radiance cache's settings."""
    _fields_ = [("enable", C.c_uint32), ("levels", C.c_uint32), ("log2_table", C.c_uint32),
                ("min_resolution", C.c_uint32), ("max_resolution", C.c_uint32),
                ("training_stride", C.c_uint32), ("training_steps", C.c_uint32), ("seed", C.c_uint32),
                ("learning_rate", C.c_float), ("terminate_bounce", C.c_uint32), ("reserved", C.c_uint32 * 2)]


CACHE_INPUTS = 64
CACHE_WEIGHTS = 21504

STRUCTS = [Geometry, Instance, Texture, TextureInput, Material, Environment, Light, SceneDesc, SceneResult,
           Target, Settings, FrameDesc, FrameResult, Options, TemporalDesc, TemporalInstance,
           CacheDesc]

# TemporalValidationSettings' defaults (temporal.hpp:28-33).
DEFAULT_VALIDATION = (0.01, 0.01, 0.9, 32.0)

# lotus_cuda_read_product's products.
PRODUCT_SURFACE = 1
PRODUCT_PREVIOUS_SURFACE = 2
PRODUCT_VALIDITY = 3
PRODUCT_RADIANCE = 4
PRODUCT_PREVIOUS_RADIANCE = 5
PRODUCT_BATCH = 6
PRODUCT_RESTIR_INITIAL = 7
PRODUCT_RESTIR_TEMPORAL = 8
PRODUCT_RESTIR_PREVIOUS = 9
PRODUCT_RESTIR_SPATIAL = 10
PRODUCT_RESTIR_SOURCES = 11
PRODUCT_RESTIR_SURFACES = 12
PRODUCT_RESTIR_PREVIOUS_SURFACES = 13
PRODUCT_FILTER = 14

try:
    import numpy as _np

    # The reference's record layouts (temporal.hpp:193-235,
    # vulkan_backend.hpp:152-178).
    TEMPORAL_PIXEL = _np.dtype([("normal_depth", "<f4", 4), ("motion_depth", "<f4", 4),
                                ("instance_id", "<u8"), ("material_id", "<u8"), ("flags", "<u4"),
                                ("albedo", "<u4"), ("shading_normal", "<u4"), ("reserved", "<u4")])
    VALIDITY_PIXEL = _np.dtype([("valid", "<u4"), ("rejection", "<u4"), ("previous_index", "<u4"),
                                ("reserved", "<u4")])
    RADIANCE_PIXEL = _np.dtype([("color", "<f4", 4), ("sample_count", "<u4"), ("moments", "<f4", 2),
                                ("variance", "<f4")])
    RESTIR_PIXEL = _np.dtype([("sample", "<u4"), ("weight_sum", "<f4"), ("selected_target", "<f4"),
                              ("candidate_count", "<u4"), ("uv", "<f4", 2), ("proposal", "<f4"),
                              ("flags", "<u4"), ("contribution", "<f4", 4)])
    RESTIR_REUSE = _np.dtype([("pixel", RESTIR_PIXEL), ("normalization", "<f4"),
                              ("supporting_candidates", "<u4"), ("previous_index", "<u4"), ("age", "<u4")])
    RESTIR_SURFACE = _np.dtype([("vectors", "<f4", (9, 4)), ("instance_id", "<u8"), ("material_id", "<u8")])
    PRODUCT_DTYPES = {
        PRODUCT_SURFACE: TEMPORAL_PIXEL, PRODUCT_PREVIOUS_SURFACE: TEMPORAL_PIXEL,
        PRODUCT_VALIDITY: VALIDITY_PIXEL, PRODUCT_RADIANCE: RADIANCE_PIXEL,
        PRODUCT_PREVIOUS_RADIANCE: RADIANCE_PIXEL, PRODUCT_BATCH: _np.dtype(("<f4", 4)),
        PRODUCT_RESTIR_INITIAL: RESTIR_PIXEL, PRODUCT_RESTIR_TEMPORAL: RESTIR_REUSE,
        PRODUCT_RESTIR_PREVIOUS: RESTIR_REUSE, PRODUCT_RESTIR_SPATIAL: RESTIR_REUSE,
        PRODUCT_RESTIR_SOURCES: _np.dtype(("<u4", 4)), PRODUCT_RESTIR_SURFACES: RESTIR_SURFACE,
        PRODUCT_RESTIR_PREVIOUS_SURFACES: RESTIR_SURFACE, PRODUCT_FILTER: _np.dtype(("<f4", 12)),
    }
except ImportError:  # pragma: no cover
    PRODUCT_DTYPES = {}


def temporal_desc(frame, current_view, previous_view=None, previous_world_to_clip=None,
                  history_available=False, accumulate_radiance=False, max_history_samples=32,
                  filter_iterations=0, validation=DEFAULT_VALIDATION, moment_precision=0):
    d = TemporalDesc()
    d.frame = frame
    d.current_view[:] = [float(v) for v in current_view]
    d.previous_view[:] = [float(v) for v in (previous_view if previous_view is not None else current_view)]
    d.previous_world_to_clip[:] = [float(v) for v in (previous_world_to_clip if previous_world_to_clip is not None
                                                     else frame.world_to_clip)]
    d.validation[:] = [float(v) for v in validation]
    d.history_available = 1 if history_available else 0
    d.accumulate_radiance = 1 if accumulate_radiance else 0
    d.max_history_samples = max_history_samples
    d.filter_iterations = filter_iterations
    d.moment_precision = moment_precision
    return d


def default_settings(**overrides):
    """PathTracingSettings' defaults (vulkan_backend.hpp:697-738)."""
    s = Settings(integrator=INTEGRATOR_REFERENCE,
                 light_sampling=LIGHT_SAMPLING_MIS,
                 sample_index=0, max_bounces=64, max_samples=0,
                 restir_candidates=8, restir_temporal=0,
                 restir_max_history_candidates=32, restir_spatial=0,
                 restir_spatial_radius=1, restir_proposal=0,
                 environment_background=0, output=OUTPUT_RADIANCE,
                 restir_spatial_neighbours=0)
    for k, v in overrides.items():
        setattr(s, k, v)
    return s


def make_frame(world_to_clip, width, height, settings=None, frame_count=1,
               clear_color=(0.0, 0.0, 0.0, 0.0), data_window=(0, 0, 0, 0),
               display_window=(0.0, 0.0, 0.0, 0.0), read_back=True, flags=0, clear_depth=1.0):
    f = FrameDesc()
    for i, v in enumerate(world_to_clip):
        f.world_to_clip[i] = float(v)
    f.target.width = width
    f.target.height = height
    for i in range(4):
        f.target.display_window[i] = display_window[i]
        f.target.data_window[i] = data_window[i]
        f.target.clear_color[i] = clear_color[i]
    f.target.read_back = 1 if read_back else 0
    f.target.clear_depth = clear_depth
    f.settings = settings if settings is not None else default_settings()
    f.frame_count = frame_count
    f.flags = flags
    return f


def check_struct_sizes(lib):
    """Raises when a ctypes mirror's size differs from the C struct's."""
    sizes = (C.c_uint64 * 32)()
    n = lib.lotus_cuda_struct_sizes(sizes, 32)
    if n != len(STRUCTS):
        raise RuntimeError(f"library reports {n} structs, bindings know {len(STRUCTS)}")
    for i, s in enumerate(STRUCTS):
        if C.sizeof(s) != sizes[i]:
            raise RuntimeError(f"{s.__name__}: ctypes {C.sizeof(s)} bytes, C {sizes[i]} bytes")
    return [int(sizes[i]) for i in range(n)]
