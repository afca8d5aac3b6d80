/* SPDX-License-Identifier: Apache-2.0
 *
 * lotus_cuda.h: the C ABI of the B200 (sm_100a) integrator backend.
 *
 * This is the drop-in boundary that stands in for the reference's
 * Vulkan backend (`lotus-render-vulkan`). A host that drives
 * `Lotus::OffscreenRenderer` (include/lotus/vulkan_backend.hpp:753-842 in the
 * reference) maps its calls onto these entry points one for one:
 *
 *   CreateOffscreenRenderer  (vulkan_backend.hpp:879-883)  -> lotus_cuda_create
 *   UpdateScene(SceneUpdate) (vulkan_backend.hpp:816-817)  -> lotus_cuda_update_scene
 *     (instance-only and point-edit updates: lotus_cuda_update_instances,
 *      lotus_cuda_update_geometry)
 *   RenderScene(...)         (vulkan_backend.hpp:789-791)  -> lotus_cuda_render
 *   RayQueryCapability()     (vulkan_backend.hpp:767)      -> lotus_cuda_capability
 *   ~OffscreenRenderer       (vulkan_backend.hpp:757)      -> lotus_cuda_destroy
 *
 * Conventions (the reference's, vulkan_backend.hpp:744-759, 812-815):
 *   - Every call returns LOTUS_PASS, LOTUS_FAIL or LOTUS_SKIP (the reference's
 *     FrameStatus) and never throws across the boundary. A detail string
 *     says why on Fail/Skip.
 *   - Invalid settings Fail without poisoning the renderer. A failed device
 *     operation poisons it: later calls Fail until it is destroyed.
 *   - Calls are synchronous, one frame in flight, one CUDA stream per
 *     renderer; a handle is not thread-safe.
 *   - The renderer owns all device memory. Input arrays are host memory,
 *     read during the call only.
 *   - Structs are plain data; matrices are column-major 4x4 floats
 *     (Lotus::Matrix4, include/lotus/render_world.hpp:16-18).
 */
#ifndef LOTUS_CUDA_H
#define LOTUS_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LOTUS_CUDA_ABI_VERSION 10u

/* FrameStatus (vulkan_backend.hpp:23-27). */
#define LOTUS_PASS 0
#define LOTUS_FAIL 1
#define LOTUS_SKIP 77

/* Integrator (vulkan_backend.hpp:639-648). */
#define LOTUS_INTEGRATOR_REFERENCE 0u
#define LOTUS_INTEGRATOR_WAVEFRONT 1u

/* LightSampling (vulkan_backend.hpp:650-670). */
#define LOTUS_LIGHT_SAMPLING_BSDF 0u
#define LOTUS_LIGHT_SAMPLING_MIS 1u
#define LOTUS_LIGHT_SAMPLING_RESTIR_INITIAL 2u

/* kMaxWavefrontBounces (vulkan_backend.hpp:694): a larger max_bounces Fails. */
#define LOTUS_MAX_BOUNCES 1024u
/* Bounces the wavefront integrator runs as rounds of extension, shading and
 * shadow kernels before its tail kernel takes the paths still queued. */
#define LOTUS_WAVEFRONT_ROUNDS 9u
/* How many per-bounce queue counts a frame result reports. */
#define LOTUS_MAX_REPORTED_BOUNCES 64u

/* UsdPreviewSurface flags (gpu_scene.hpp:82-87). */
#define LOTUS_MATERIAL_SPECULAR_WORKFLOW 1u
#define LOTUS_MATERIAL_THIN_WALLED 2u

/* ShadingModel (material.hpp:90-99): the material's surface model. */
#define LOTUS_MODEL_PREVIEW_SURFACE 0u
#define LOTUS_MODEL_GLTF_PBR 1u

/* One mesh: Lotus::MeshGeometry (render_world.hpp:39-58), object space. */
typedef struct lotus_geometry {
  const float* positions;     /* 3 floats per vertex */
  const uint32_t* triangles;  /* 3 vertex indices per triangle */
  const float* normals;       /* NULL, or 9 floats per triangle: corner normals */
  uint32_t vertex_count;
  uint32_t triangle_count;
  /* Texture-coordinate sets (MeshGeometry::texcoords, in key order): set k's
   * (s, t) of triangle i's corner c at texcoords[6 * (k * triangle_count +
   * i) + 2 * c]; NULL when texcoord_sets is 0. */
  const float* texcoords;
  uint32_t texcoord_sets;
  /* Colour sets (MeshGeometry::colors, in key order): linear RGB, finite,
   * unclamped; set k holds color_counts[k] RGB values, 3 * triangle_count
   * (one per triangle corner, triangle by triangle) or 1 (the whole mesh),
   * the sets one after another in `colors`. NULL when color_sets is 0. */
  uint32_t color_sets;
  const float* colors;
  const uint32_t* color_counts;
} lotus_geometry;

/* One placed mesh: SceneUpdate's instance (extraction.hpp:313-354). */
typedef struct lotus_instance {
  float world_from_object[16]; /* column-major; the last row must be 0 0 0 1 */
  uint32_t geometry;           /* index into lotus_scene_desc::geometries */
  uint32_t material;           /* index into lotus_scene_desc::materials */
  /* The texture-coordinate set its material's lookups read (SceneInstance::
   * texcoords, extraction.hpp:44-48): k > 0 for its geometry's set k - 1,
   * LOTUS_NO_TEXCOORDS (0) for the material's texcoord_fallback. */
  uint32_t texcoord_set;
  /* The colour set its UsdPreviewSurface material's base colour reads
   * (SceneInstance::colors, extraction.hpp:49-51): k > 0 for its geometry's
   * set k - 1, clamped into [0, 1], LOTUS_NO_COLORS (0) for the material's
   * own base colour. A base-colour texture lookup wins; glTF PBR reads no
   * colour set. */
  uint32_t color_set;
} lotus_instance;

/* Zero in every index field below means "none", so that a zeroed struct
 * holds the defaults: no texture-coordinate set, no image, no lookup. */
#define LOTUS_NO_TEXCOORDS 0u
#define LOTUS_NO_COLORS 0u

/* TextureFormat (material.hpp:15-23): texels of 4 bytes (8-bit channels,
 * the sRGB format's red, green and blue sRGB-encoded, alpha linear) or of
 * 16 (four floats). */
#define LOTUS_TEXTURE_RGBA8_UNORM 0u
#define LOTUS_TEXTURE_RGBA8_SRGB 1u
#define LOTUS_TEXTURE_RGBA32_FLOAT 2u

/* A decoded image (material.hpp:29-40): rows from the top of the image,
 * texture coordinates (0, 0) its bottom-left corner. */
typedef struct lotus_texture {
  const void* texels;
  uint32_t width;
  uint32_t height;
  uint32_t format;      /* LOTUS_TEXTURE_* */
  uint32_t reserved;
} lotus_texture;

/* TextureWrap (material.hpp:42-50). */
#define LOTUS_WRAP_BLACK 0u   /* transparent black */
#define LOTUS_WRAP_CLAMP 1u   /* the nearest edge texel */
#define LOTUS_WRAP_REPEAT 2u
#define LOTUS_WRAP_MIRROR 3u

#define LOTUS_NO_TEXTURE 0u

/* A texture lookup that drives one material input (TextureInput,
 * material.hpp:52-74): the texture filtered bilinearly at
 * (m0 s + m1 t + m2, m3 s + m4 t + m5) of the material's texture
 * coordinates, times scale plus bias; `fallback`, unscaled, when `texture`
 * is LOTUS_NO_TEXTURE (a key naming no image). */
typedef struct lotus_texture_input {
  uint32_t texture;      /* k > 0: lotus_scene_desc::textures[k - 1]; LOTUS_NO_TEXTURE (0) */
  uint32_t channel;      /* 0..3, a scalar input's channel */
  uint32_t wrap_s;       /* LOTUS_WRAP_* */
  uint32_t wrap_t;
  float scale[4];
  float bias[4];
  float fallback[4];
  float st_transform[6];
  uint32_t reserved[2];
} lotus_texture_input;

/* A material's texture-input slots (material.hpp:262-286): a lookup
 * replaces the input's constant, clamped into its range (the normal slots'
 * into [-1, 1]: a tangent-space normal, in the frame of the texture
 * coordinates' differentials about the interpolated shading normal).
 * Slots 0 and 1 are the geometry's in every model; the others are
 * numbered per model. */
#define LOTUS_SLOT_OPACITY 0u
#define LOTUS_SLOT_NORMAL 1u
/* UsdPreviewSurface's. */
#define LOTUS_SLOT_BASE_COLOR 2u
#define LOTUS_SLOT_ROUGHNESS 3u
#define LOTUS_SLOT_METALLIC 4u
#define LOTUS_SLOT_EMISSION 5u
#define LOTUS_SLOT_SPECULAR_COLOR 6u
/* glTF PBR's. */
#define LOTUS_GLTF_SLOT_BASE_COLOR 2u
#define LOTUS_GLTF_SLOT_METALLIC 3u
#define LOTUS_GLTF_SLOT_ROUGHNESS 4u
#define LOTUS_GLTF_SLOT_EMISSIVE 5u
#define LOTUS_GLTF_SLOT_SPECULAR 6u
#define LOTUS_GLTF_SLOT_SPECULAR_COLOR 7u
#define LOTUS_GLTF_SLOT_TRANSMISSION 8u
#define LOTUS_GLTF_SLOT_CLEARCOAT 9u
#define LOTUS_GLTF_SLOT_CLEARCOAT_ROUGHNESS 10u
#define LOTUS_GLTF_SLOT_CLEARCOAT_NORMAL 11u
#define LOTUS_GLTF_SLOT_SHEEN_COLOR 12u
#define LOTUS_GLTF_SLOT_SHEEN_ROUGHNESS 13u
#define LOTUS_TEXTURE_SLOTS 14u
#define LOTUS_NO_LOOKUP 0u

/* A material (material.hpp:219-245): its surface model's constants,
 * UsdPreviewSurface's (material.hpp:137-173) or MaterialX's glTF PBR
 * surface's (material.hpp:180-217), plus its coverage (material.hpp:
 * 103-116). The first fields serve both models: base_color, roughness,
 * metallic, emission (glTF PBR's emissive), specular_color, ior and
 * transmission carry the inputs of those names; transmission_color and
 * flags are UsdPreviewSurface's only, and the fields after `normal` glTF
 * PBR's only. */
typedef struct lotus_material {
  float base_color[3];
  float roughness;
  float emission[3];
  float metallic;
  float specular_color[3];
  float ior;
  float transmission_color[3];
  float transmission;
  float opacity;            /* surface coverage in [0, 1] */
  float opacity_threshold;  /* > 0: binary coverage */
  uint32_t flags;           /* LOTUS_MATERIAL_* */
  uint32_t model;           /* LOTUS_MODEL_* */
  /* Per LOTUS_SLOT_*: k > 0 for lotus_scene_desc::texture_inputs[k - 1],
   * LOTUS_NO_LOOKUP (0) for the constant. */
  uint32_t lookups[LOTUS_TEXTURE_SLOTS];
  /* The texture coordinates on an instance with no set
   * (MaterialGeometry::texcoord_fallback). */
  float texcoord_fallback[2];
  /* The tangent-space shading normal (MaterialGeometry::normal, in
   * [-1, 1]); all zero means the identity (0, 0, 1). A normal-map lookup
   * (LOTUS_SLOT_NORMAL) replaces it. */
  float normal[3];
  /* glTF PBR: a finite, non-negative factor on emissive. */
  float emissive_strength;
  /* glTF PBR, each in [0, 1]: the dielectric reflection's weight, the
   * clearcoat's weight and roughness. */
  float specular;
  float clearcoat;
  float clearcoat_roughness;
  /* glTF PBR: the sheen's colour (each in [0, 1]; the largest is its
   * weight) and roughness in [0, 1]. */
  float sheen_color[3];
  float sheen_roughness;
} lotus_material;

/* A latitude-longitude environment image (render_world.hpp:122-133): RGBA
 * float texels, rows from the top. The renderer builds its sampling
 * distribution (gpu_scene.cpp:620-711). */
typedef struct lotus_environment {
  const float* texels;              /* 4 floats per texel, width*height texels */
  uint32_t width;
  uint32_t height;
  float scale[3];                   /* multiplies the texels' RGB */
  float environment_from_world[9];  /* rows: the image frame's unit axes in world space */
} lotus_environment;

/* LightShape (render_world.hpp:79-84). */
#define LOTUS_LIGHT_SPHERE 0u
#define LOTUS_LIGHT_RECT 1u
#define LOTUS_LIGHT_DISK 2u
#define LOTUS_LIGHT_DISTANT 3u

/* An analytic light: Lotus::Light (render_world.hpp:86-114). It only emits:
 * it neither reflects nor blocks light, and camera rays do not see it. A
 * sphere is centred on its frame's origin, its radius scaled by the cube
 * root of the frame's absolute determinant; a rect or disk lies in its
 * frame's XY plane and emits from its -Z side; a distant light shines along
 * its frame's -Z axis, a parallel light when its angle is 0. */
typedef struct lotus_light {
  uint32_t shape;               /* LOTUS_LIGHT_* */
  uint32_t normalize;           /* UsdLux normalize: radiance over area / size factor */
  float world_from_light[16];   /* column-major */
  float radiance[3];            /* linear RGB; a parallel light's irradiance */
  float radius;                 /* sphere, disk */
  float width;                  /* rect extent along X */
  float height;                 /* rect extent along Y */
  float angle;                  /* distant: angular diameter in degrees */
  uint32_t reserved;
} lotus_light;

/* The whole scene. Slot 0 of materials is the default material. */
typedef struct lotus_scene_desc {
  const lotus_geometry* geometries;
  const lotus_instance* instances;
  const lotus_material* materials;
  const lotus_environment* environment; /* NULL: no environment image */
  uint32_t geometry_count;
  uint32_t instance_count;
  uint32_t material_count;
  float environment_constant[3];  /* the constant environment radiance */
  const lotus_light* lights;      /* analytic lights (the snapshot's Light list); NULL if none */
  uint32_t light_count;
  /* The images and lookups the materials' texture inputs name. */
  const lotus_texture* textures;
  uint32_t texture_count;
  uint32_t texture_input_count;
  const lotus_texture_input* texture_inputs;
} lotus_scene_desc;

/* GpuSceneEvidence, in part. */
typedef struct lotus_scene_result {
  int32_t status;
  uint32_t triangle_count;      /* unique triangles over all geometries */
  uint32_t instance_count;
  uint32_t light_count;         /* light table entries */
  uint32_t bvh_node_count;      /* BLAS nodes over all geometries */
  uint32_t tlas_node_count;
  double build_gpu_ms;          /* device LBVH builds and table uploads */
  uint64_t device_bytes;        /* scene bytes resident on the device */
  char detail[256];
} lotus_scene_result;

/* OffscreenTarget (vulkan_backend.hpp:253-282). */
typedef struct lotus_target {
  uint32_t width;
  uint32_t height;
  float display_window[4];   /* {x, y, w, h}; w or h <= 0 means the whole image */
  int32_t data_window[4];    /* {x, y, w, h}; w or h <= 0 means the whole image */
  float clear_color[4];
  uint32_t read_back;        /* 0 keeps the frame on the device */
  float clear_depth;         /* Vulkan window depth in [0, 1] of the depth product's clears (OffscreenTarget's 1) */
} lotus_target;

/* PathTracingSettings (vulkan_backend.hpp:697-738). */
typedef struct lotus_settings {
  uint32_t integrator;        /* LOTUS_INTEGRATOR_* */
  uint32_t light_sampling;    /* LOTUS_LIGHT_SAMPLING_* */
  uint32_t sample_index;
  uint32_t max_bounces;
  uint32_t max_samples;       /* 0: no limit */
  uint32_t restir_candidates;
  uint32_t restir_temporal;
  uint32_t restir_max_history_candidates;
  uint32_t restir_spatial;
  uint32_t restir_spatial_radius;
  uint32_t restir_proposal;
  uint32_t environment_background;
  uint32_t output;            /* LOTUS_OUTPUT_* (SceneOutput) */
  /* The spatial pass's neighbours. 0: the reference's four axis neighbours
   * at restir_spatial_radius (restir.slang:402-410). 1..8: that many
   * distinct pixels drawn uniformly from the disk of that radius around the
   * pixel (the pixel itself excluded), from their own random stream. No
   * counterpart in the reference. */
  uint32_t restir_spatial_neighbours;
} lotus_settings;

/* The most neighbours a disk-mode spatial pass draws. */
#define LOTUS_MAX_SPATIAL_NEIGHBOURS 8u

/* lotus_settings::output (SceneOutput, vulkan_backend.hpp:617-634): the
 * accumulated path-traced radiance, or a diagnostic of the pixel centre's
 * closest hit (not accumulated; misses keep the clear colour): its
 * barycentric weights (1 - b1 - b2, b1, b2, 1), the world-space shading
 * normal, the base colour with alpha 1, or (roughness, metallic, 0, 1). */
#define LOTUS_OUTPUT_RADIANCE 0u
#define LOTUS_OUTPUT_BARYCENTRICS 1u
#define LOTUS_OUTPUT_SHADING_NORMAL 2u
#define LOTUS_OUTPUT_ALBEDO 3u
#define LOTUS_OUTPUT_ROUGHNESS_METALLIC 4u

/* lotus_frame_desc::flags. TIMINGS times the kernels of the call's last
 * sample by class (the reference's WavefrontTimings, vulkan_backend.hpp:
 * 52-68). COUNT_VISITS makes the last sample count BVH nodes, triangles and
 * instances visited per ray kind (slower; for roofline accounting). */
#define LOTUS_FRAME_TIMINGS 1u
#define LOTUS_FRAME_COUNT_VISITS 2u
/* DEPTH writes the D32 depth product (vulkan_backend.hpp:230, 769-773; the
 * camera pass, path_trace.slang:69-97): the pixel centre's closest hit,
 * traced with the fixed coverage sequence of sample 0, as Vulkan window
 * depth (clip z / clip w through the frame's camera); pixels without a hit
 * and outside the data window keep target.clear_depth, or with DEPTH_KEEP
 * (OffscreenTarget::clear_depth_enabled false) the preceding frame's depth.
 * lotus_cuda_read_depth copies it. */
#define LOTUS_FRAME_DEPTH 4u
#define LOTUS_FRAME_DEPTH_KEEP 8u

/* One RenderScene call: DrawSummary::world_to_clip in the OpenGL clip
 * convention (extraction.hpp:23), the target and the settings. */
typedef struct lotus_frame_desc {
  float world_to_clip[16];
  lotus_target target;
  lotus_settings settings;
  uint32_t frame_count;
  uint32_t flags;   /* LOTUS_FRAME_* */
} lotus_frame_desc;

/* GpuFrameEvidence (vulkan_backend.hpp:202-249), in part. */
typedef struct lotus_frame_result {
  int32_t status;
  uint32_t frames_rendered;
  uint32_t samples_per_pixel;
  uint32_t wavefront_rounds;
  uint64_t completion;
  /* Rays traced by this call, over all its samples. */
  uint64_t camera_rays;
  uint64_t extension_rays;
  uint64_t shadow_rays;
  /* Device time of the call's samples (CUDA events), readback excluded. */
  double gpu_ms;
  /* Queue occupancy of the last sample: per bounce, paths that entered the
   * ray queue; element 0 is the camera rays. wavefront_rounds: the bounces
   * run as extension and shading rounds; with max_bounces above
   * LOTUS_WAVEFRONT_ROUNDS the tail kernel follows the paths still queued
   * after them (their rays count at the bounce they leave from). */
  uint32_t wavefront_path_counts[LOTUS_MAX_REPORTED_BOUNCES];
  uint32_t wavefront_path_count_size;
  /* With LOTUS_FRAME_TIMINGS: device time of the last sample's kernels, by
   * class (wavefront integrator; the megakernel reports camera_gpu_ms). */
  uint32_t timings_available;
  double camera_gpu_ms;
  double extend_gpu_ms;
  double shade_gpu_ms;
  double shadow_gpu_ms;
  double resolve_gpu_ms;
  uint32_t extend_launches;
  uint32_t shadow_launches;
  /* With LOTUS_FRAME_COUNT_VISITS: the last sample's visits, indexed
   * camera, extension, shadow; rays[k] is the ray count they cover. */
  uint64_t visit_rays[3];
  uint64_t node_visits[3];
  uint64_t triangle_visits[3];
  uint64_t instance_visits[3];
  /* With the radiance cache: the last sample's cache kernels (inference,
   * training, Adam) with LOTUS_FRAME_TIMINGS, and the sample's queries and
   * training records. */
  double cache_gpu_ms;
  uint32_t cache_queries;
  uint32_t cache_training_records;
  /* With LOTUS_FRAME_TIMINGS: the tail kernel's device time (the paths still
   * queued after the wavefront_rounds rounds, each followed to its end). */
  double tail_gpu_ms;
  /* The samples the call's last wavefront held: a call that adds two or
   * more samples (without the radiance cache) runs them in waves of eight
   * (lotus_cuda_options::samples_per_wave; halved while the call adds fewer)
   * to a wavefront, and then the queue counts, the timings and the visit
   * counts above are those of its last wave, its samples together. */
  uint32_t last_wave_samples;
  uint32_t reserved;
  /* With LOTUS_FRAME_TIMINGS: the device time spent putting the extension
   * queues of bounces 1 and on in key order (origin cell, direction
   * octant) before their rounds; the shading pass that queues the rays
   * writes their keys. */
  double sort_gpu_ms;
  /* With LOTUS_FRAME_TIMINGS and the radiance cache: cache_gpu_ms split
   * into inference (the queries put in spatial order, then the network's
   * forward pass) and training (targets, training passes, Adam). */
  double cache_infer_gpu_ms;
  double cache_train_gpu_ms;
  char detail[256];
} lotus_frame_result;

typedef struct lotus_cuda_options {
  int32_t device;          /* CUDA device ordinal */
  uint32_t flags;          /* reserved, 0 */
  uint32_t bvh_leaf_size;  /* most triangles per BLAS leaf, 1..8; 0: the default (1) */
  /* Launch shape of the persistent extension and shadow kernels (0: the
   * defaults): a warp's idle lanes take new rays when fewer than
   * trace_refill_below (1..32) of its lanes still hold one, and at most
   * trace_blocks_per_sm blocks run on each SM. */
  uint32_t trace_refill_below;
  uint32_t trace_blocks_per_sm;
  /* Bounces the wavefront integrator runs as rounds before its tail kernel
   * takes the paths still queued (1..LOTUS_MAX_BOUNCES + 1). 0: RenderScene
   * chooses them from its first sample of each scene and frame shape (run
   * with LOTUS_WAVEFRONT_ROUNDS): the first bounce whose queue held fewer
   * paths than the extension kernel keeps resident on the device at once
   * (at least 65536); other calls use LOTUS_WAVEFRONT_ROUNDS. Results do not
   * depend on it. */
  uint32_t wavefront_rounds;
  /* A BVH walk's step budget (node visits, leaf tests and instance entries);
   * 0: 2^18, which only a corrupt BVH could need. A walk that runs out of it,
   * or whose traversal stack overflows, makes its frame Fail with a detail
   * naming the cause and poisons the renderer. Tests lower it to make the
   * bound run out. */
  uint32_t traversal_step_limit;
  /* Samples a RenderScene call that adds several runs in one wavefront
   * (their paths side by side in one set of queues, so that each launch
   * pays its ramp-up and drain once for all of them): 1, 2, 4 or 8; 0: 8.
   * The path state and queues take this many times the target's pixels.
   * Results do not depend on it. */
  uint32_t samples_per_wave;
} lotus_cuda_options;

typedef struct lotus_cuda_renderer lotus_cuda_renderer;

/* The library's ABI version (LOTUS_CUDA_ABI_VERSION). Needs no GPU. */
uint32_t lotus_cuda_abi_version(void);

/* sizeof of each struct above, in declaration order, so a binding can check
 * its mirrors. Writes at most `capacity` sizes; returns how many there are.
 * Needs no GPU. */
uint32_t lotus_cuda_struct_sizes(uint64_t* sizes, uint32_t capacity);

/* RayQueryCapability (vulkan_backend.hpp:767): LOTUS_PASS when an sm_100
 * device is present, LOTUS_SKIP with the reason otherwise. */
int32_t lotus_cuda_capability(int32_t device, char* detail, size_t detail_size);

/* CreateOffscreenRenderer (vulkan_backend.hpp:879-883). */
int32_t lotus_cuda_create(const lotus_cuda_options* options,
    lotus_cuda_renderer** renderer, char* error, size_t error_size);

void lotus_cuda_destroy(lotus_cuda_renderer* renderer);

/* UpdateScene (vulkan_backend.hpp:816-817): replaces the resident scene.
 * Builds the BVHs on the device (binned SAH per geometry, all geometries in
 * one launch, LBVH above 65,536 triangles; binned SAH or LBVH over the
 * instances; each collapsed to a 4-wide BVH), the light table and the
 * environment distribution. Restarts the accumulation. A scene holds fewer
 * than 2^28 triangles. */
int32_t lotus_cuda_update_scene(lotus_cuda_renderer* renderer,
    const lotus_scene_desc* scene, lotus_scene_result* result);

/* UpdateScene with a SceneUpdate that changes instances only (transform
 * edits, material slots; vulkan_backend.cpp's TLAS-only update path): the
 * resident scene's instances become `instances` (any count, naming its
 * geometries and materials). Rebuilds the light table, the instance records
 * and the TLAS; the BLASes, materials and environment stay. Restarts the
 * accumulation. Invalid instances Fail without poisoning; the scene is
 * unchanged then. build_gpu_ms counts the uploads and builds. */
int32_t lotus_cuda_update_instances(lotus_cuda_renderer* renderer,
    const lotus_instance* instances, uint32_t count, lotus_scene_result* result);

/* UpdateScene with a compatible point edit of one geometry (its triangles
 * and vertex count kept; the reference refits, gpu_scene.cpp:2303-2322):
 * the resident geometry `geometry` takes new positions (and new corner
 * normals, which a geometry with corner normals must be given and one
 * without must not). Refits that geometry's BLAS in place (its topology
 * kept, its boxes recomputed bottom-up from the new positions), then
 * rebuilds the light table, instance records and TLAS. Restarts the
 * accumulation. The images equal those of lotus_cuda_update_scene with the
 * edited scene (hits are decided by triangle tests alone). */
int32_t lotus_cuda_update_geometry(lotus_cuda_renderer* renderer, uint32_t geometry,
    const float* positions, uint32_t vertex_count, const float* normals, lotus_scene_result* result);

/* RenderScene (vulkan_backend.hpp:789-791), Radiance output: adds
 * frame_count samples per pixel (up to max_samples) to the accumulation and
 * writes its mean. With target.read_back and a non-NULL `color`, copies the
 * RGBA32F colour (width*height*4 floats, top-left rows) into `color`. */
int32_t lotus_cuda_render(lotus_cuda_renderer* renderer,
    const lotus_frame_desc* frame, lotus_frame_result* result, float* color);

/* TemporalFrameSettings (include/lotus/temporal.hpp:58-98) and the
 * snapshot cameras of one RenderTemporalScene call
 * (vulkan_backend.hpp:807-810). The host keeps the reference's
 * TemporalHistory (temporal.hpp:112-125) and says whether it kept the
 * preceding frame. */
typedef struct lotus_temporal_desc {
  lotus_frame_desc frame;            /* this frame's camera, target and settings */
  float current_view[16];            /* Camera::view of this frame */
  float previous_view[16];           /* the preceding frame's Camera::view */
  float previous_world_to_clip[16];  /* the preceding frame's projection * view, OpenGL clip */
  float validation[4];               /* absolute depth, relative depth, min normal cosine, max motion (px) */
  uint32_t history_available;        /* TemporalFrame::previous is present */
  uint32_t accumulate_radiance;
  uint32_t max_history_samples;      /* 1..65536 when accumulating */
  uint32_t filter_iterations;        /* 0..8; needs accumulate_radiance */
  uint32_t history_rectification;    /* TemporalHistoryRectification; only None (0) is built */
  /* Precision of the luminance moments the temporal accumulation keeps
   * between frames. LOTUS_MOMENTS_FP32: as the reference. LOTUS_MOMENTS_FP16:
   * the first moment and the central second moment (m2 - m1^2, which keeps
   * the variance from cancelling away) are rounded to half precision
   * (saturating at 65504) where the reference stores the moments, the blend
   * itself staying FP32; the record keeps the reference's 32-byte layout,
   * and the radiance products give the raw second moment back. No
   * counterpart in the reference. */
  uint32_t moment_precision;
} lotus_temporal_desc;

#define LOTUS_MOMENTS_FP32 0u
#define LOTUS_MOMENTS_FP16 1u

/* One instance's temporal identity (the reference's TemporalInstanceRecord,
 * backend/vulkan/temporal_metadata.hpp), in scene instance order. */
typedef struct lotus_temporal_instance {
  float previous_world_from_object[16];
  uint64_t instance_id;
  uint64_t material_id;
  uint32_t flags;     /* 2: rigid correspondence with the preceding frame, 4: unchanged material */
  uint32_t reserved;
} lotus_temporal_instance;

/* Replaces the instances' temporal identities. Until called after a scene
 * update, each instance's ids are its index and material slot, its previous
 * transform its current one, and its flags 6. */
int32_t lotus_cuda_set_temporal_instances(lotus_cuda_renderer* renderer,
    const lotus_temporal_instance* instances, uint32_t count);

/* RenderTemporalScene (vulkan_backend.hpp:807-810): the primary-surface
 * metadata and its reprojection; with RestirInitial light sampling the
 * ReSTIR DI initial, temporal (restir_temporal) and spatial (restir_spatial)
 * reservoir passes; one fresh batch of frame_count samples whose primary
 * direct light is the final reservoir's; and with accumulate_radiance the
 * SVGF accumulation, variance and filter_iterations a-trous iterations into
 * the colour. */
int32_t lotus_cuda_render_temporal(lotus_cuda_renderer* renderer,
    const lotus_temporal_desc* temporal, lotus_frame_result* result, float* color);

/* Temporal products (the reference's TemporalProducts and RestirProducts,
 * vulkan_backend.hpp:90-200), read back from the device. */
#define LOTUS_PRODUCT_SURFACE 1u            /* TemporalPixel, 64 B/pixel, this frame */
#define LOTUS_PRODUCT_PREVIOUS_SURFACE 2u   /* TemporalPixel, the preceding frame */
#define LOTUS_PRODUCT_VALIDITY 3u           /* TemporalValidityPixel, 16 B/pixel */
#define LOTUS_PRODUCT_RADIANCE 4u           /* TemporalRadiancePixel, 32 B/pixel */
#define LOTUS_PRODUCT_PREVIOUS_RADIANCE 5u
#define LOTUS_PRODUCT_BATCH 6u              /* the fresh batch's RGBA mean, 16 B/pixel */
#define LOTUS_PRODUCT_RESTIR_INITIAL 7u     /* RestirPixel, 48 B/pixel */
#define LOTUS_PRODUCT_RESTIR_TEMPORAL 8u    /* RestirReusePixel, 64 B/pixel */
#define LOTUS_PRODUCT_RESTIR_PREVIOUS 9u
#define LOTUS_PRODUCT_RESTIR_SPATIAL 10u
#define LOTUS_PRODUCT_RESTIR_SOURCES 11u    /* 4 u32 per pixel */
#define LOTUS_PRODUCT_RESTIR_SURFACES 12u   /* 160 B/pixel */
#define LOTUS_PRODUCT_RESTIR_PREVIOUS_SURFACES 13u
#define LOTUS_PRODUCT_FILTER 14u            /* 3 float4 per pixel: two ping-pong halves, guides */

/* Copies a product of the latest temporal frame into `out`; returns the
 * bytes copied, or -1 when the product does not exist or does not fit. */
int64_t lotus_cuda_read_product(lotus_cuda_renderer* renderer, uint32_t product, void* out,
    uint64_t capacity_bytes);

/* The colour of the latest frame into host memory (width*height*4 floats). */
int32_t lotus_cuda_read_color(lotus_cuda_renderer* renderer, float* color,
    uint64_t capacity_floats);

/* ReadBackScene (vulkan_backend.hpp:819-821), for validation: copies of the
 * resident scene as the device holds it, decoded into this ABI's records.
 * `what` selects the copy and `index` the geometry where one is meant:
 *   LOTUS_SCENE_POSITIONS  geometry `index`'s positions, 3 floats per vertex
 *   LOTUS_SCENE_TRIANGLES  its triangles, 3 vertex indices each
 *   LOTUS_SCENE_NORMALS    its corner normals, 9 floats per triangle (none
 *                          without them)
 *   LOTUS_SCENE_INSTANCES  every instance: lotus_instance records from the
 *                          device's instance records (world_from_object,
 *                          geometry, material slot)
 *   LOTUS_SCENE_MATERIALS  every material: lotus_material records from the
 *                          device's material table
 *   LOTUS_SCENE_ENVIRONMENT the constant environment radiance, 3 floats
 * Returns the bytes the copy takes (with `out` NULL, without copying), or
 * -1 without a scene or for an unknown selection or a short buffer. */
#define LOTUS_SCENE_POSITIONS 1u
#define LOTUS_SCENE_TRIANGLES 2u
#define LOTUS_SCENE_NORMALS 3u
#define LOTUS_SCENE_INSTANCES 4u
#define LOTUS_SCENE_MATERIALS 5u
#define LOTUS_SCENE_ENVIRONMENT 6u
int64_t lotus_cuda_read_scene(lotus_cuda_renderer* renderer, uint32_t what, uint32_t index, void* out,
    uint64_t capacity_bytes);

/* The depth product of the latest RenderScene frame that asked for it
 * (LOTUS_FRAME_DEPTH) into host memory: width*height floats, top-left rows.
 * Fail when the latest frame wrote none. */
int32_t lotus_cuda_read_depth(lotus_cuda_renderer* renderer, float* depth, uint64_t capacity_floats);

/* The renderer's CUDA stream (a cudaStream_t), for callers that time its
 * work with their own events. */
void* lotus_cuda_stream(lotus_cuda_renderer* renderer);

/* The light table as the device holds it (GpuLightRecord, gpu_scene.hpp:
 * 120-126): 4 words per entry {pdf, threshold, alias, instance}, then the
 * per-instance first entries. Returns the entry count, or -1. */
int64_t lotus_cuda_read_light_table(lotus_cuda_renderer* renderer,
    uint32_t* records, uint64_t record_capacity, uint32_t* offsets,
    uint64_t offset_capacity);

/* The most pixels lotus_cuda_render_static renders. */
#define LOTUS_STATIC_MAX_PIXELS 65536u

/* Renders a frame without allocating device memory. No counterpart in the
 * reference: its Vulkan renderer always allocates its own targets.
 *
 * For hosts that cannot call cudaMalloc when they want a frame: a delegate
 * inside another framework's frame loop that owns every allocation, or a
 * real-time caller that must not block in the allocator. The frame's
 * scratch (path state, queues, accumulation, counters) lives in one
 * file-scope device array of about 12 MB that every GPU which loads the
 * library holds until the process exits. The caller passes the renderer
 * (whose resident scene is the input), the frame, and `color_device`:
 * device memory for width*height*4 floats, which receives the RGBA32F mean
 * of frame_count samples from settings.sample_index (top-left rows; pixels
 * outside the data window get the clear colour). Each call starts its own
 * accumulation; none carries over. settings.max_samples, when nonzero,
 * caps the samples added as RenderScene's does for a fresh accumulation.
 *
 * Limits: at most LOTUS_STATIC_MAX_PIXELS pixels (larger targets Fail with
 * that reason); Radiance with BSDF or MIS light sampling; a renderer whose
 * radiance cache is configured on Fails (this entry point never uses the
 * cache, so its image would not be RenderScene's). All calls share the one
 * scratch array, which keeps the last call's contents, so calls whose GPU
 * work overlaps (other threads or streams) race and corrupt each other.
 * The first call on each device looks up the array's address with that
 * device current; make it before any stream capture (a cudaDeviceReset
 * invalidates that address together with every renderer on the device).
 * A launch or device error Fails the call and poisons the renderer, as
 * lotus_cuda_render does. Calls no cudaMalloc, cudaFree or allocating
 * library routine. */
int32_t lotus_cuda_render_static(lotus_cuda_renderer* renderer,
    const lotus_frame_desc* frame, float* color_device, lotus_frame_result* result);

/* ------------------------------------------------------------------------
 * Batched rendering. No counterpart in the reference: up to
 * LOTUS_BATCH_MAX_SCENES independent scenes, each with its own target,
 * rendered as one wavefront (one camera launch over all their pixels, then
 * per bounce one extension, shading and shadow launch over all their
 * queued paths), a sample captured as one CUDA graph. Each scene is built
 * as lotus_cuda_update_scene builds one; each frame renders as
 * lotus_cuda_render would render it (the same images, bit for bit), with
 * the wavefront integrator, Bsdf or Mis light sampling and no max_samples. */

#define LOTUS_BATCH_MAX_SCENES 64u

typedef struct lotus_cuda_batch lotus_cuda_batch;

/* options: the device and the persistent kernels' launch shape. */
int32_t lotus_cuda_batch_create(const lotus_cuda_options* options,
    lotus_cuda_batch** batch, char* error, size_t error_size);

void lotus_cuda_batch_destroy(lotus_cuda_batch* batch);

/* Replaces the batch's scenes; results[k] (if not NULL) for scene k. */
int32_t lotus_cuda_batch_set_scenes(lotus_cuda_batch* batch,
    const lotus_scene_desc* scenes, uint32_t count, lotus_scene_result* results);

/* The batch's launch shape, for a tuner (0 picks each default): the
 * persistent kernels' refill threshold and blocks per SM (as
 * lotus_cuda_options' trace_* fields), the wavefront rounds before the tail
 * kernel (as lotus_cuda_options::wavefront_rounds), and the camera pass's
 * order within each scene: LOTUS_CAMERA_TILE_ROWS (the image's rows) or
 * warp tiles of 4x8, 8x4 or 16x2 pixels (where every scene's size is a
 * multiple of the tile; rows otherwise). Results do not depend on any of
 * them. */
#define LOTUS_CAMERA_TILE_ROWS 1u
#define LOTUS_CAMERA_TILE_4X8 2u
#define LOTUS_CAMERA_TILE_8X4 3u
#define LOTUS_CAMERA_TILE_16X2 4u
int32_t lotus_cuda_batch_set_tuning(lotus_cuda_batch* batch,
    uint32_t trace_refill_below, uint32_t trace_blocks_per_sm, uint32_t wavefront_rounds, uint32_t camera_tile);

/* frames[k] renders scene k (count = the batch's scene count, every
 * frame_count equal). A scene's accumulation continues while its frame
 * description is unchanged. results[k] and colors[k] (host memory, W x H x 4
 * floats, or NULL) are per scene; `total` (if not NULL) holds the rays and
 * device time of the whole call. */
int32_t lotus_cuda_batch_render(lotus_cuda_batch* batch,
    const lotus_frame_desc* frames, uint32_t count, lotus_frame_result* results,
    float* const* colors, lotus_frame_result* total);

/* ------------------------------------------------------------------------
 * Learned radiance cache. No counterpart in the reference: a hash-grid
 * encoded MLP (five 64-wide ReLU layers, RGB out; BF16 on the tensor cores,
 * FP32 accumulation) trained online on the wavefront path tracer's own
 * radiance. With the cache enabled, wavefront paths end into it at their
 * second vertex, after next event estimation there (the cache stands for
 * the light the vertex scatters besides its direct light), except one path
 * in `training_stride`, which is traced in full and trains it on what it
 * gathered after that vertex's emission and shadow ray. */

#define LOTUS_CACHE_INPUTS 64u
#define LOTUS_CACHE_WEIGHTS 21504u  /* 5 x 64 x 64 + 64 x 16 FP32 */

typedef struct lotus_cache_desc {
  uint32_t enable;           /* 1: paths end into the cache; 0: plain PT */
  uint32_t levels;           /* hash-grid levels, 1..16 (0: 16) */
  uint32_t log2_table;       /* entries per level, log2, 10..22 (0: 19) */
  uint32_t min_resolution;   /* coarsest grid resolution (0: 16) */
  uint32_t max_resolution;   /* finest grid resolution (0: 2048) */
  uint32_t training_stride;  /* one path in this many trains the cache (0: 32) */
  uint32_t training_steps;   /* Adam steps per sample (0: 1) */
  uint32_t seed;             /* weight and grid initialisation */
  float learning_rate;       /* Adam step size (0: 1e-2) */
  /* The bounce whose vertex the paths end into the cache at, 1..16 (0: 1,
   * the second vertex). A later vertex shrinks the cache's bias in the
   * image by the throughput of the bounces before it, at the cost of
   * tracing them. */
  uint32_t terminate_bounce;
  uint32_t reserved[2];
} lotus_cache_desc;

/* (Re)creates the cache over the resident scene's bounds (a unit box
 * without a scene) with fresh weights, and sets whether RenderScene's
 * wavefront samples use it. Restarts the accumulation. */
int32_t lotus_cuda_configure_cache(lotus_cuda_renderer* renderer,
    const lotus_cache_desc* desc, char* detail, size_t detail_size);

/* The network's FP32 weights (LOTUS_CACHE_WEIGHTS floats; layer l < 5 is
 * W[in][out] 64 x 64, layer 5 is 64 x 16 with RGB in its first three
 * columns): read (write == 0) or replaced (write != 0). */
int32_t lotus_cuda_cache_weights(lotus_cuda_renderer* renderer, float* weights,
    uint64_t count, int32_t write);

/* Network outputs (n x 3, host memory) for encoded inputs (n x 64). */
int32_t lotus_cuda_cache_infer(lotus_cuda_renderer* renderer,
    const float* inputs, uint32_t n, float* outputs);

/* Gradients of the relative L2 loss sum_s,c (y - t)^2 / (y^2 + 0.01), the
 * denominator held constant, over encoded inputs (n x 64) and targets
 * (n x 3): weight gradients (LOTUS_CACHE_WEIGHTS), input gradients
 * (n x 64) and the loss. Any output may be NULL. Leaves the weights as
 * they are. */
int32_t lotus_cuda_cache_gradient(lotus_cuda_renderer* renderer,
    const float* inputs, const float* targets, uint32_t n, float* weight_grad,
    float* input_grad, float* loss);

/* The network inputs (n x 64) of raw records (n x 16 floats: position,
 * roughness; direction, 0; normal, 0; albedo, 0). */
int32_t lotus_cuda_cache_encode(lotus_cuda_renderer* renderer,
    const float* records, uint32_t n, float* inputs);

/* `steps` training steps on raw records (n x 16 floats, as above) and RGB
 * targets (n x 3): each runs the training pass over all n records (the
 * gradients of the relative L2 loss reaching the weights and the hash
 * grid) and one Adam step. losses[k] (if not NULL) is the summed loss
 * before step k. */
int32_t lotus_cuda_cache_train(lotus_cuda_renderer* renderer,
    const float* records, const float* targets, uint32_t n, uint32_t steps,
    float* losses);

#ifdef __cplusplus
}
#endif

#endif /* LOTUS_CUDA_H */
