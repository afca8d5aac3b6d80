// SPDX-License-Identifier: Apache-2.0
// The GPU scene as the kernels read it, and software ray traversal.
//
// B200 has no RT cores, so the reference's ray queries (TraceRayInline over
// a driver-built TLAS/BLAS, backend/vulkan/shaders/common/scene.slang:
// 424-460 in hydra-lotus) become a two-level BVH walk:
//   - one BLAS per geometry in object space, one TLAS over the instances'
//     world boxes; all BLAS nodes share one pool and all triangles another;
//   - 128-byte 4-wide nodes holding the children's boxes by axis and
//     bound, so one node is seven 16-byte loads and tests four children;
//   - triangles stored in leaf order as three float4 corners in a 64-byte
//     record, the original primitive index in the first corner's w;
//   - instance records split by use: a traversal record (object-from-world
//     rows, BLAS root, flags) and a shading record (world-from-object rows,
//     material, light-table offset, normals).
// Triangles are intersected with the watertight test of Woop, Benthin and
// Wald (JCGT 2013) in object space. Equal hit distances resolve to the
// smaller (instance, primitive), so the closest hit does not depend on the
// traversal order.
#pragma once

#include "../../include/lotus_cuda.h"
#include "common.cuh"

namespace lotus {

// Child encoding: >= 0 an interior node index in the same pool; < 0 a leaf
// whose first primitive is ~child (a triangle-pool index in a BLAS, an
// instance in the TLAS) with `count` primitives.
constexpr int32_t kEmptyChild = 0x7FFFFFFF;
constexpr int32_t kExitInstance = 0x7FFFFFFE;
constexpr int kStackSize = 128;
// A walk that takes more steps than this (SceneView::step_limit, unless a
// test lowers it) ends early: only a corrupt BVH could need it, and the
// bound keeps such a walk from spinning. A walk that ends on its step
// limit, or that had to drop a child because its stack was full, reports
// itself through SceneView::walk_failure, and the frame Fails.
constexpr uint32_t kMaxTraversalSteps = 1u << 18;
// Set in Walk::steps when a child did not fit on the stack: the walk then
// counts as out of steps, ends at its next pop and reports the overflow.
constexpr uint32_t kWalkOverflow = 1u << 31;
// SceneView::walk_failure[1] bits: a walk ran out of steps; a walk's stack
// overflowed.
constexpr uint32_t kWalkFailedSteps = 1u;
constexpr uint32_t kWalkFailedStack = 2u;

// Triangle records are four float4 (64 bytes, cache-sector aligned): three
// object-space corners, the primitive index in the first corner's w.
constexpr int kTriStride = 4;
// Bits of a BLAS leaf reference that hold its triangle count less one
// (leaves hold 1..8 triangles); the rest hold the first triangle, so a
// scene holds fewer than 2^28 triangles.
constexpr uint32_t kLeafCountBits = 3;
constexpr uint32_t kMaxSceneTriangles = 1u << 28;

// The traversal's 4-wide node: four children's boxes by axis and bound
// (component i is child i) and their references: a node index, or for a
// BLAS leaf ~(first triangle << kLeafCountBits | count - 1), for a TLAS
// leaf ~instance; `count` keeps the leaves' triangle counts. 128 bytes.
struct alignas(16) Bvh4Node {
  float4 lo_x, hi_x, lo_y, hi_y, lo_z, hi_z;
  int4 child;
  int4 count;
};
static_assert(sizeof(Bvh4Node) == 128, "4-wide node is 128 bytes");

struct alignas(16) BvhNode {
  float4 x;   // child 0 low, child 0 high, child 1 low, child 1 high (x axis)
  float4 y;
  float4 z;
  int4 c;     // child 0, child 1, child 0 count, child 1 count
};
static_assert(sizeof(BvhNode) == 64, "BVH node is 64 bytes");

// Per instance, read at TLAS leaves.
struct alignas(16) InstanceTraversal {
  float4 inv[3];   // object_from_world rows
  uint32_t blas_root;  // BLAS pool index of the geometry's root, or kEmptyChild
  uint32_t flags;      // bit 0: every surface is opaque
  uint32_t material;
  uint32_t light_offset;  // first light-table entry, or kNoLights
};
static_assert(sizeof(InstanceTraversal) == 64, "traversal record is 64 bytes");

// Per instance, read at shading.
struct alignas(16) InstanceShading {
  float4 m[3];     // world_from_object rows: (m[0], m[4], m[8], m[12]), ...
  uint32_t material;
  uint32_t light_offset;
  uint32_t normals;    // first corner-normal triple of the geometry, or kNoLights
  uint32_t mirror;     // the linear part's determinant is negative
};
static_assert(sizeof(InstanceShading) == 64, "shading record is 64 bytes");

constexpr uint32_t kInstanceOpaque = 1u;

// lotus_material as seven float4. The fields marked glTF hold MaterialX's
// glTF PBR inputs on a material of that model (kMaterialGltf).
struct alignas(16) MaterialRecord {
  float4 base_roughness;       // base colour, roughness
  float4 emission_metallic;    // emission (glTF: emissive), metallic
  float4 specular_ior;         // specular colour, ior
  float4 transmission;         // transmission colour (glTF: unused), transmission
  float4 coverage;             // opacity, threshold, flags (bits), glTF: the dielectric's f0
  float4 gltf;                 // glTF: specular, clearcoat, clearcoat roughness, emissive strength
  float4 sheen;                // glTF: sheen colour, sheen roughness
};
static_assert(sizeof(MaterialRecord) == 112, "material record is 112 bytes");

// MaterialRecord::coverage.z flag bits the renderer adds to the material's
// own LOTUS_MATERIAL_* bits: some input has a texture lookup; the opacity
// has one.
constexpr uint32_t kMaterialTextured = 1u << 8;
constexpr uint32_t kMaterialOpacityTextured = 1u << 9;
// The material is MaterialX's glTF PBR surface (LOTUS_MODEL_GLTF_PBR).
constexpr uint32_t kMaterialGltf = 1u << 10;
// kMaterialTextured is set too for a constant tangent-space normal other
// than (0, 0, 1), which MaterialLookups::normal holds.

// A texture input (TextureInputRecord, scene.slang:44-55): the texture's
// index (kNoTexture: the fallback), channel and wrap modes, then scale,
// bias and fallback, and the lookup's coordinate rows
// (s' = st_s.x s + st_s.y t + st_s.z, t' likewise).
struct alignas(16) TextureLookup {
  uint32_t texture;
  uint32_t channel;
  uint32_t wrap_s;
  uint32_t wrap_t;
  float4 scale;
  float4 bias;
  float4 fallback;
  float4 st_s;
  float4 st_t;
};
static_assert(sizeof(TextureLookup) == 96, "TextureLookup is 96 bytes");
constexpr uint32_t kNoTexture = 0xFFFFFFFFu;

// A material's lookups per texture slot (kNoTexture: its constant) and its
// texture-coordinate fallback.
struct alignas(16) MaterialLookups {
  uint32_t slot[LOTUS_TEXTURE_SLOTS];
  float fallback_s;
  float fallback_t;
  float normal[3];  // the constant tangent-space normal
  uint32_t reserved;
};
static_assert(sizeof(MaterialLookups) == 80, "MaterialLookups is 80 bytes");

// A light-table entry (GpuLightRecord, gpu_scene.hpp:120-126).
struct alignas(16) LightRecord {
  float pdf;
  float threshold;
  uint32_t alias;
  uint32_t instance;
};

// One analytic light in world space (GpuAnalyticLightRecord,
// gpu_scene.hpp:144-166): a sphere's centre and radius; a rect's or disk's
// centre, half axes and emitting-side unit normal with its area in w; a
// distant light's unit direction towards it in axis_u with 1 - cos of its
// cone in w; the radiance with the light's table probability in w.
struct alignas(16) AnalyticLight {
  float4 position;
  float4 axis_u;
  float4 axis_v;
  float4 normal;
  float4 radiance;
  uint32_t shape;
  uint32_t reserved[3];
};
static_assert(sizeof(AnalyticLight) == 96, "AnalyticLight is 96 bytes");

// One interior node of the binary crossing hierarchy over the sphere, rect
// and disk lights (GpuLightNode, gpu_scene.hpp:174-186): each child's box,
// the child's bits in low.w.
struct alignas(16) LightNode {
  float4 low0, high0, low1, high1;
};
static_assert(sizeof(LightNode) == 64, "LightNode is 64 bytes");

struct SceneView {
  const Bvh4Node* __restrict__ tlas;
  const Bvh4Node* __restrict__ blas;
  const float4* __restrict__ tris;          // kTriStride per leaf-ordered triangle
  const InstanceTraversal* __restrict__ inst_trav;
  const InstanceShading* __restrict__ inst_shade;
  const MaterialRecord* __restrict__ materials;
  const float* __restrict__ normals;        // 9 floats per original triangle
  const LightRecord* __restrict__ lights;
  const float4* __restrict__ light_verts;   // 3 world corners per light entry
  const float4* __restrict__ light_radiance;// emission * coverage per light entry
  const float4* __restrict__ env_texels;
  const float* __restrict__ env_floats;     // density, marginal, conditional
  const uint32_t* __restrict__ env_guide;   // guide tables of the marginal and each conditional
  uint32_t instance_count;
  uint32_t light_count;
  uint32_t env_bound;
  uint32_t env_width, env_height, env_columns, env_rows;
  float env_selection;
  float env_scale[3];
  float env_frame[9];       // rows of environment_from_world
  float env_constant[3];
  const AnalyticLight* __restrict__ analytic;  // every analytic record, table entry or not
  const LightNode* __restrict__ light_nodes;   // the crossing hierarchy (node 0: root)
  const uint32_t* __restrict__ distant;        // indices of the distant lights
  uint32_t analytic_count;
  uint32_t light_node_count;
  uint32_t distant_count;
  uint32_t step_limit;       // a walk's step budget (kMaxTraversalSteps)
  uint32_t full_shading;     // some material has a texture lookup, a mapped normal or the glTF PBR model
  const float* __restrict__ albedo_tables;  // the composed closure's (albedo.cuh), 76800 floats
  // Texture lookups: every texture's texels decoded to linear RGBA, one
  // after another; per texture its first texel, width and height; the
  // scene's texture inputs; per material its lookups (read only for
  // kMaterialTextured materials); every geometry's texture-coordinate sets,
  // three (s, t) per triangle; per instance the first coordinate of its
  // set (kNoTexture: the material's fallback).
  const float4* __restrict__ tex_texels;
  const uint4* __restrict__ tex_info;
  const TextureLookup* __restrict__ lookups;
  const MaterialLookups* __restrict__ mat_lookups;
  const float2* __restrict__ texcoords;
  const uint32_t* __restrict__ inst_texcoords;
  const float* __restrict__ colors;        // colour sets, RGB
  const uint2* __restrict__ inst_colors;   // per instance: (first float, whole-mesh flag) or kNoTexture
  // Two words the renderer clears before and reads after each frame: the
  // number of walks that failed and the kWalkFailed* bits of their causes.
  uint32_t* walk_failure;
};

// Buckets of the environment distribution's guide tables (powers of two):
// the marginal's, then each row's conditional's, kEnv* + 1 entries each.
constexpr uint32_t kEnvGuideMarginal = 1024;
constexpr uint32_t kEnvGuideConditional = 512;

struct Hit {
  uint32_t instance;
  uint32_t tri;        // leaf-ordered triangle-pool index
  float b1, b2;
  float t;
};

// One texel of a lookup's texture at integer coordinates (x, y), rows from
// the top, after each axis's wrap (the Vulkan sampler address modes the
// reference binds, vulkan_backend.cpp:3038-3053): transparent black outside
// the image, the edge texel, the coordinate modulo the size, or mirrored
// every size texels.
__device__ __forceinline__ int32_t wrap_texel(int32_t i, int32_t n, uint32_t mode) {
  if (mode == LOTUS_WRAP_CLAMP) return i < 0 ? 0 : (i >= n ? n - 1 : i);
  if (mode == LOTUS_WRAP_REPEAT) {
    const int32_t r = i % n;
    return r < 0 ? r + n : r;
  }
  if (mode == LOTUS_WRAP_MIRROR) {
    int32_t r = i % (2 * n);
    if (r < 0) r += 2 * n;
    return r < n ? r : 2 * n - 1 - r;
  }
  return (i < 0 || i >= n) ? -1 : i;
}

__device__ __forceinline__ float4 texel_at(const SceneView& S, const uint4& info, int32_t x, int32_t y,
    uint32_t wrap_s, uint32_t wrap_t) {
  const int32_t xi = wrap_texel(x, (int32_t)info.y, wrap_s);
  const int32_t yi = wrap_texel(y, (int32_t)info.z, wrap_t);
  if (xi < 0 || yi < 0) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  return S.tex_texels[info.x + (uint32_t)yi * info.y + (uint32_t)xi];
}

// Lookup (scene.slang:315-328): the bilinear texel at (s, t) (texel centres
// at (i + 1/2) / size, rows from the image's top), times scale plus bias;
// the unscaled fallback when the input names no image.
__device__ __forceinline__ float4 texture_lookup(const SceneView& S, const TextureLookup& L, float s, float t) {
  if (L.texture == kNoTexture) return L.fallback;
  const float u = L.st_s.x * s + L.st_s.y * t + L.st_s.z;
  const float v = 1.0f - (L.st_t.x * s + L.st_t.y * t + L.st_t.z);
  const uint4 info = S.tex_info[L.texture];
  // Far outside the image every wrap mode reads a defined texel; keep the
  // integer conversion in range.
  const float x = fminf(fmaxf(u * (float)info.y - 0.5f, -16777216.0f), 16777216.0f);
  const float y = fminf(fmaxf(v * (float)info.z - 0.5f, -16777216.0f), 16777216.0f);
  const float fx = floorf(x), fy = floorf(y);
  const float ax = x - fx, ay = y - fy;
  const int32_t ix = (int32_t)fx, iy = (int32_t)fy;
  const float4 t00 = texel_at(S, info, ix, iy, L.wrap_s, L.wrap_t);
  const float4 t10 = texel_at(S, info, ix + 1, iy, L.wrap_s, L.wrap_t);
  const float4 t01 = texel_at(S, info, ix, iy + 1, L.wrap_s, L.wrap_t);
  const float4 t11 = texel_at(S, info, ix + 1, iy + 1, L.wrap_s, L.wrap_t);
  const float bx = 1.0f - ax, by = 1.0f - ay;
  const float4 top = make_float4(t00.x * bx + t10.x * ax, t00.y * bx + t10.y * ax, t00.z * bx + t10.z * ax,
      t00.w * bx + t10.w * ax);
  const float4 bottom = make_float4(t01.x * bx + t11.x * ax, t01.y * bx + t11.y * ax, t01.z * bx + t11.z * ax,
      t01.w * bx + t11.w * ax);
  const float4 f = make_float4(top.x * by + bottom.x * ay, top.y * by + bottom.y * ay, top.z * by + bottom.z * ay,
      top.w * by + bottom.w * ay);
  return make_float4(f.x * L.scale.x + L.bias.x, f.y * L.scale.y + L.bias.y, f.z * L.scale.z + L.bias.z,
      f.w * L.scale.w + L.bias.w);
}

__device__ __forceinline__ float lookup_channel(const float4& v, uint32_t channel) {
  return channel == 0 ? v.x : channel == 1 ? v.y : channel == 2 ? v.z : v.w;
}

// HitTexcoords (scene.slang:362-374): the instance's set interpolated with
// the barycentrics, or the material's fallback.
__device__ __forceinline__ void hit_texcoords(const SceneView& S, uint32_t instance, const MaterialLookups& ml,
    uint32_t primitive, float b1, float b2, float& s, float& t) {
  const uint32_t base = S.inst_texcoords[instance];
  if (base == kNoTexture) {
    s = ml.fallback_s;
    t = ml.fallback_t;
    return;
  }
  const float2* c = S.texcoords + base + 3 * (size_t)primitive;
  const float2 t0 = c[0], t1 = c[1], t2 = c[2];
  s = t0.x + b1 * (t1.x - t0.x) + b2 * (t2.x - t0.x);
  t = t0.y + b1 * (t1.y - t0.y) + b2 * (t2.y - t0.y);
}

// The opacity lookup's channel at a hit, saturated (0 where the lookup
// overflows). Not inlined: the walks that meet textured coverage are rare,
// and its registers stay out of the traversal kernels.
static __device__ __noinline__ float textured_opacity(const SceneView& S, uint32_t material, uint32_t instance,
    uint32_t primitive, float b1, float b2) {
  const MaterialLookups ml = S.mat_lookups[material];
  float s, t;
  hit_texcoords(S, instance, ml, primitive, b1, b2, s, t);
  const TextureLookup& L = S.lookups[ml.slot[LOTUS_SLOT_OPACITY]];
  const float opacity = lookup_channel(texture_lookup(S, L, s, t), L.channel);
  return isfinite(opacity) ? fminf(fmaxf(opacity, 0.0f), 1.0f) : 0.0f;
}

// Coverage (scene.slang:393-406): the material's opacity, or its lookup's
// channel at the hit; 0 or 1 under a threshold.
__device__ __forceinline__ float material_coverage(const SceneView& S, const MaterialRecord& m, uint32_t material,
    uint32_t instance, uint32_t primitive, float b1, float b2) {
  float opacity = m.coverage.x;
  if (__float_as_uint(m.coverage.z) & kMaterialOpacityTextured)
    opacity = textured_opacity(S, material, instance, primitive, b1, b2);
  const float threshold = m.coverage.y;
  if (threshold > 0.0f) return opacity >= threshold ? 1.0f : 0.0f;
  return opacity;
}

// kFullShading false: the scene has no textured coverage (SceneView::full_shading
// clear), and the walk compiles without the lookup.
template <bool kFullShading = true>
__device__ __forceinline__ float instance_coverage(const SceneView& S, uint32_t instance, uint32_t primitive,
    float b1, float b2) {
  const uint32_t material = S.inst_trav[instance].material;
  const MaterialRecord& m = S.materials[material];
  if (!kFullShading) {
    if (m.coverage.y > 0.0f) return m.coverage.x >= m.coverage.y ? 1.0f : 0.0f;
    return m.coverage.x;
  }
  return material_coverage(S, m, material, instance, primitive, b1, b2);
}

__device__ __forceinline__ F3 safe_inverse(F3 d) {
  auto inv = [](float x) {
    return 1.0f / (fabsf(x) > 1e-30f ? x : (x < 0.0f ? -1e-30f : 1e-30f));
  };
  return V(inv(d.x), inv(d.y), inv(d.z));
}

// The reciprocal direction of the walks' slab tests, with the hardware's
// approximate reciprocal (a few ulps): a slab test's far distance carries a
// relative margin of 2^-18, far above that error, so boxes are still never
// culled where a triangle test could accept a hit. The exact safe_inverse
// stays where a box test decides a result (the light hierarchy's crossings).
__device__ __forceinline__ F3 slab_inverse(F3 d) {
  auto inv = [](float x) {
    const float y = fabsf(x) > 1e-30f ? x : (x < 0.0f ? -1e-30f : 1e-30f);
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(y));
    return r;
  };
  return V(inv(d.x), inv(d.y), inv(d.z));
}

// Read-only loads of the BVH and triangle pools that ask L1 to keep their
// lines over the path state's streaming accesses (evict_last).
__device__ __forceinline__ float4 ld_keep(const float4* p) {
  float4 v;
  asm("ld.global.nc.L1::evict_last.v4.f32 {%0,%1,%2,%3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
  return v;
}
__device__ __forceinline__ int4 ld_keep_i(const int4* p) {
  int4 v;
  asm("ld.global.nc.L1::evict_last.v4.s32 {%0,%1,%2,%3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p));
  return v;
}
// A node's boxes and child references; interior visits never read `count`.
__device__ __forceinline__ Bvh4Node load_node(const Bvh4Node* p) {
  Bvh4Node n;
  n.lo_x = ld_keep(&p->lo_x); n.hi_x = ld_keep(&p->hi_x);
  n.lo_y = ld_keep(&p->lo_y); n.hi_y = ld_keep(&p->hi_y);
  n.lo_z = ld_keep(&p->lo_z); n.hi_z = ld_keep(&p->hi_z);
  n.child = ld_keep_i(&p->child);
  n.count = make_int4(0, 0, 0, 0);
  return n;
}

struct WatertightRay {
  F3 org;
  uint32_t axes;  // kx | ky << 2 | kz << 4
  float sx, sy, sz;
};

__device__ __forceinline__ WatertightRay prepare_ray(F3 org, F3 dir) {
  WatertightRay w;
  w.org = org;
  const float ax = fabsf(dir.x), ay = fabsf(dir.y), az = fabsf(dir.z);
  const int kz = ax > ay ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
  int kx = kz == 2 ? 0 : kz + 1;
  int ky = kx == 2 ? 0 : kx + 1;
  if (component(dir, kz) < 0.0f) {
    const int s = kx;
    kx = ky;
    ky = s;
  }
  const float dz = component(dir, kz);
  w.axes = (uint32_t)kx | (uint32_t)ky << 2 | (uint32_t)kz << 4;
  w.sx = component(dir, kx) / dz;
  w.sy = component(dir, ky) / dz;
  w.sz = 1.0f / dz;
  return w;
}

__device__ __forceinline__ bool intersect_triangle(const WatertightRay& r, F3 v0, F3 v1, F3 v2,
    float& t, float& b1, float& b2) {
  const int kx = r.axes & 3u, ky = (r.axes >> 2) & 3u, kz = r.axes >> 4;
  const F3 A = v0 - r.org, B = v1 - r.org, C = v2 - r.org;
  const float Akz = component(A, kz), Bkz = component(B, kz), Ckz = component(C, kz);
  const float Ax = component(A, kx) - r.sx * Akz;
  const float Ay = component(A, ky) - r.sy * Akz;
  const float Bx = component(B, kx) - r.sx * Bkz;
  const float By = component(B, ky) - r.sy * Bkz;
  const float Cx = component(C, kx) - r.sx * Ckz;
  const float Cy = component(C, ky) - r.sy * Ckz;
  float U = Cx * By - Cy * Bx;
  float W1 = Ax * Cy - Ay * Cx;
  float W2 = Bx * Ay - By * Ax;
  if (U == 0.0f || W1 == 0.0f || W2 == 0.0f) {
    U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
    W1 = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
    W2 = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
  }
  if ((U < 0.0f || W1 < 0.0f || W2 < 0.0f) && (U > 0.0f || W1 > 0.0f || W2 > 0.0f)) return false;
  const float det = U + W1 + W2;
  if (det == 0.0f) return false;
  const float Az = r.sz * Akz, Bz = r.sz * Bkz, Cz = r.sz * Ckz;
  const float T = U * Az + W1 * Bz + W2 * Cz;
  const float rcp = 1.0f / det;
  t = T * rcp;
  b1 = W1 * rcp;
  b2 = W2 * rcp;
  return true;
}

// Slab tests of a 4-wide node's children against [tmin, tmax]. The far
// distance gets a relative margin of 2^-18 (the clamp to tmax included), so
// a box is never culled where the triangle test, whose distances carry
// their own rounding, could still accept a hit: hits are decided by
// triangle tests alone, whatever the BVH's shape.
__device__ __forceinline__ float slab_near(float lo, float hi, float o, float inv, float& far) {
  const float a = (lo - o) * inv, b = (hi - o) * inv;
  far = fmaxf(a, b);
  return fminf(a, b);
}

__device__ __forceinline__ void test_children4(const Bvh4Node& n, F3 o, F3 inv, float tmin, float tmax,
    float tn[4], bool hit[4]) {
  const float lx[4] = {n.lo_x.x, n.lo_x.y, n.lo_x.z, n.lo_x.w}, hx[4] = {n.hi_x.x, n.hi_x.y, n.hi_x.z, n.hi_x.w};
  const float ly[4] = {n.lo_y.x, n.lo_y.y, n.lo_y.z, n.lo_y.w}, hy[4] = {n.hi_y.x, n.hi_y.y, n.hi_y.z, n.hi_y.w};
  const float lz[4] = {n.lo_z.x, n.lo_z.y, n.lo_z.z, n.lo_z.w}, hz[4] = {n.hi_z.x, n.hi_z.y, n.hi_z.z, n.hi_z.w};
  const int c[4] = {n.child.x, n.child.y, n.child.z, n.child.w};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    float fx, fy, fz;
    const float nx = slab_near(lx[i], hx[i], o.x, inv.x, fx);
    const float ny = slab_near(ly[i], hy[i], o.y, inv.y, fy);
    const float nz = slab_near(lz[i], hz[i], o.z, inv.z, fz);
    const float t0 = fmaxf(fmaxf(nx, ny), fmaxf(nz, tmin));
    const float t1 = fminf(fminf(fx, fy), fminf(fz, tmax));
    tn[i] = t0;
    hit[i] = t0 <= t1 + fabsf(t1) * 3.8146973e-6f && c[i] != kEmptyChild;
  }
}

__device__ __forceinline__ F3 row_point(const float4* r, F3 p) {
  return V(r[0].x * p.x + r[0].y * p.y + r[0].z * p.z + r[0].w,
           r[1].x * p.x + r[1].y * p.y + r[1].z * p.z + r[1].w,
           r[2].x * p.x + r[2].y * p.y + r[2].z * p.z + r[2].w);
}

__device__ __forceinline__ F3 row_vector(const float4* r, F3 d) {
  return V(r[0].x * d.x + r[0].y * d.y + r[0].z * d.z,
           r[1].x * d.x + r[1].y * d.y + r[1].z * d.z,
           r[2].x * d.x + r[2].y * d.y + r[2].z * d.z);
}

struct TraversalCounters {
  uint32_t nodes;
  uint32_t triangles;
  uint32_t instances;
};

// The traversal state of one ray over the two-level 4-wide BVH. Walks are
// made of four kinds of work: an interior node's slab tests (its hit
// children pushed nearest last, the nearest taken next), one BLAS leaf's
// triangle tests, an instance's entry and the exit marker. kAnyHit walks
// are the shadow query of ShadowTransmittance (scene.slang:445-460); the
// others find the closest accepted hit of Trace (scene.slang:424-439), whose
// coverage tests draw from the path's random state. TLAS leaves (one
// instance each) go on the stack like nodes, and entering one pushes a
// marker that restores the world-space ray when popped.
struct Walk {
  F3 origin, direction;  // the world-space ray
  F3 inv;                // 1 / direction in the current space
  WatertightRay w;       // the ray in the current space (w.org its origin)
  float tmin, best, transmittance;
  uint32_t instance, best_instance, best_tri;
  float b1, b2;
  int32_t cur;           // the next reference to process, or kWalkDone
  int32_t leaf;          // a postponed BLAS leaf, or 0
  uint32_t steps;
  int sp;
  bool found, in_blas, opaque;
};

// The walk's stack lives beside it (a local array of kStackSize entries),
// so that the walk's scalars stay in registers.
typedef int32_t WalkStack[kStackSize];

constexpr int32_t kWalkDone = 0x7FFFFFFD;

__device__ __forceinline__ void walk_begin(const SceneView& S, Walk& W, F3 origin, F3 direction,
    float tmin, float tmax) {
  W.origin = origin;
  W.direction = direction;
  W.inv = slab_inverse(direction);
  W.w.org = origin;
  W.tmin = tmin;
  W.best = tmax;
  W.transmittance = 1.0f;
  W.found = false;
  W.in_blas = false;
  W.opaque = true;
  W.instance = 0;
  W.sp = 0;
  W.steps = 0;
  W.leaf = 0;
  W.cur = S.instance_count != 0 ? 0 : kWalkDone;
}

__device__ __forceinline__ Hit walk_hit(const Walk& W) {
  Hit h;
  h.instance = W.best_instance;
  h.tri = W.best_tri;
  h.b1 = W.b1;
  h.b2 = W.b2;
  h.t = W.best;
  return h;
}

__device__ __forceinline__ bool walk_at_node(const Walk& W) { return W.cur >= 0 && W.cur < kWalkDone; }

// The next reference from the stack, or kWalkDone (also once the walk has
// used its step budget, or overflowed its stack).
__device__ __forceinline__ void walk_pop(const SceneView& S, Walk& W, const WalkStack& stack) {
  W.cur = (W.sp > 0 && W.steps < S.step_limit) ? stack[--W.sp] : kWalkDone;
}

// A walk that has ended: if it ended on its step budget or a stack
// overflow, its hits may be incomplete; count it and record the cause.
__device__ __forceinline__ void walk_check_end(const SceneView& S, const Walk& W) {
  if (W.steps >= S.step_limit) {
    atomicAdd(&S.walk_failure[0], 1u);
    atomicOr(&S.walk_failure[1], (W.steps & kWalkOverflow) ? kWalkFailedStack : kWalkFailedSteps);
  }
}

// Slab tests of the node at W.cur. Its hit children go on the stack
// (nearest last) and the nearest becomes W.cur; with none hit, W.cur is
// popped.
template <bool kCount>
__device__ __forceinline__ void walk_visit_node(const SceneView& S, Walk& W, WalkStack& stack,
    TraversalCounters* counters) {
  const Bvh4Node n = load_node(W.in_blas ? S.blas + W.cur : S.tlas + W.cur);
  if (kCount) ++counters->nodes;
  ++W.steps;
  float tn[4];
  bool h[4];
  test_children4(n, W.w.org, W.inv, W.tmin, W.best, tn, h);
  float key[4];
  int32_t ref[4] = {n.child.x, n.child.y, n.child.z, n.child.w};
#pragma unroll
  for (int i = 0; i < 4; ++i) key[i] = h[i] ? tn[i] : INFINITY;
#define LOTUS_CSWAP(a, b)                                    \
  if (key[b] < key[a]) {                                     \
    const float tk = key[a]; key[a] = key[b]; key[b] = tk;   \
    const int32_t tr = ref[a]; ref[a] = ref[b]; ref[b] = tr; \
  }
  LOTUS_CSWAP(0, 1) LOTUS_CSWAP(2, 3) LOTUS_CSWAP(0, 2) LOTUS_CSWAP(1, 3) LOTUS_CSWAP(1, 2)
#undef LOTUS_CSWAP
  if (key[0] == INFINITY) {
    walk_pop(S, W, stack);
    return;
  }
#pragma unroll
  for (int i = 3; i >= 1; --i)
    if (key[i] != INFINITY) {
      if (W.sp < kStackSize) stack[W.sp++] = ref[i];
      else W.steps |= kWalkOverflow;
    }
  W.cur = W.steps < S.step_limit ? ref[0] : kWalkDone;
}

// The triangle tests of BLAS leaf `leaf` (a negative reference). Returns
// true when an any-hit walk has met an opaque surface.
template <bool kAnyHit, bool kCount, bool kFullShading = true>
__device__ __forceinline__ bool walk_test_leaf(const SceneView& S, Walk& W, int32_t leaf, uint32_t& rng,
    TraversalCounters* counters) {
  const uint32_t code = ~(uint32_t)leaf;
  const uint32_t first = code >> kLeafCountBits;
  const uint32_t count = (code & ((1u << kLeafCountBits) - 1u)) + 1u;
  ++W.steps;
  for (uint32_t k = 0; k < count; ++k) {
    const float4* tv = S.tris + kTriStride * (size_t)(first + k);
    const float4 a = ld_keep(tv), b = ld_keep(tv + 1), cc = ld_keep(tv + 2);
    if (kCount) ++counters->triangles;
    float t, b1, b2;
    if (!intersect_triangle(W.w, V(a), V(b), V(cc), t, b1, b2)) continue;
    if (!(t >= W.tmin) || !(t <= W.best)) continue;
    const uint32_t prim = __float_as_uint(a.w);
    if (kAnyHit) {
      const float coverage = W.opaque ? 1.0f : instance_coverage<kFullShading>(S, W.instance, prim, b1, b2);
      if (coverage >= 1.0f) {
        W.found = true;
        W.transmittance = 0.0f;
        return true;
      }
      if (coverage > 0.0f) W.transmittance *= 1.0f - coverage;
    } else {
      if (W.found && t == W.best &&
          (W.instance > W.best_instance ||
           (W.instance == W.best_instance && prim >= __float_as_uint(S.tris[kTriStride * (size_t)W.best_tri].w))))
        continue;
      if (!W.opaque) {
        const float coverage = instance_coverage<kFullShading>(S, W.instance, prim, b1, b2);
        if (coverage <= 0.0f) continue;
        if (coverage < 1.0f && !(next_random(rng) < coverage)) continue;
      }
      W.found = true;
      W.best = t;
      W.best_instance = W.instance;
      W.best_tri = first + k;
      W.b1 = b1;
      W.b2 = b2;
    }
  }
  return false;
}

// W.cur is not an interior node: the exit marker, a BLAS leaf (tested
// here), or a TLAS leaf (entered). Leaves W.cur at the next reference.
// Returns true when an any-hit walk has met an opaque surface.
template <bool kAnyHit, bool kCount, bool kFullShading = true>
__device__ __forceinline__ bool walk_other(const SceneView& S, Walk& W, WalkStack& stack, uint32_t& rng,
    TraversalCounters* counters) {
  const int32_t cur = W.cur;
  if (cur == kExitInstance) {
    W.in_blas = false;
    W.w.org = W.origin;
    W.inv = slab_inverse(W.direction);
  } else if (W.in_blas) {
    if (walk_test_leaf<kAnyHit, kCount, kFullShading>(S, W, cur, rng, counters)) return true;
  } else {
    const uint32_t instance = ~(uint32_t)cur;
    if (kCount) ++counters->instances;
    ++W.steps;
    const InstanceTraversal rec = S.inst_trav[instance];
    if (rec.blas_root != (uint32_t)kEmptyChild && W.sp >= kStackSize) W.steps |= kWalkOverflow;
    if (rec.blas_root != (uint32_t)kEmptyChild && W.sp < kStackSize) {
      stack[W.sp++] = kExitInstance;
      const F3 o = row_point(rec.inv, W.origin);
      const F3 d = row_vector(rec.inv, W.direction);
      W.inv = slab_inverse(d);
      W.w = prepare_ray(o, d);
      W.instance = instance;
      W.opaque = (rec.flags & kInstanceOpaque) != 0;
      W.in_blas = true;
      W.cur = (int32_t)rec.blas_root;
      return false;
    }
  }
  walk_pop(S, W, stack);
  return false;
}

// The whole walk in one call (for kernels with one ray per thread).
template <bool kAnyHit, bool kCount, bool kFullShading = true>
__device__ __forceinline__ float traverse(const SceneView& S, F3 origin, F3 direction, float tmin,
    float tmax, uint32_t& rng, Hit& hit, bool& found, TraversalCounters* counters = nullptr) {
  Walk W;
  WalkStack stack;
  walk_begin(S, W, origin, direction, tmin, tmax);
  while (W.cur != kWalkDone) {
    if (walk_at_node(W)) {
      walk_visit_node<kCount>(S, W, stack, counters);
    } else if (walk_other<kAnyHit, kCount, kFullShading>(S, W, stack, rng, counters)) {
      break;
    }
  }
  walk_check_end(S, W);
  found = W.found;
  if (!kAnyHit && W.found) hit = walk_hit(W);
  return kAnyHit ? W.transmittance : 0.0f;
}

// Interior-node steps of a round stop once fewer lanes than this are at an
// interior node while others wait with other work: the remaining lanes
// carry their nodes into the next round instead of running the step
// nearly alone.
constexpr int kRoundNodeLanes = 8;

// One round of a warp's walks (for persistent kernels; every lane of the
// warp calls it, `active` lanes hold a walk). Interior nodes first, each
// lane postponing the first BLAS leaf it meets and carrying on, until no
// lane is left at an interior node, or fewer than kRoundNodeLanes are and
// another lane has other work; then every postponed leaf is tested, and
// finally each lane not at an interior node takes its exit marker, further
// leaf or instance entry. Each kind of work thus runs once per round over
// all the lanes that have it. Returns true for a lane whose walk has ended.
template <bool kAnyHit, bool kCount, bool kFullShading = true>
__device__ __forceinline__ bool walk_round(const SceneView& S, Walk& W, WalkStack& stack, uint32_t& rng,
    bool active, TraversalCounters* counters) {
  constexpr unsigned kAll = 0xFFFFFFFFu;
  for (;;) {
    const bool node = active && walk_at_node(W);
    const unsigned at_node = __ballot_sync(kAll, node);
    if (at_node == 0) break;
    if (__popc(at_node) < kRoundNodeLanes && __any_sync(kAll, active && !node)) break;
    if (node) {
      walk_visit_node<kCount>(S, W, stack, counters);
      if (W.in_blas && W.cur < 0 && W.leaf == 0) {
        W.leaf = W.cur;
        walk_pop(S, W, stack);
      }
    }
  }
  bool ended = false;
  const bool leaf = active && W.leaf != 0;
  if (__any_sync(kAll, leaf) && leaf) {
    ended = walk_test_leaf<kAnyHit, kCount, kFullShading>(S, W, W.leaf, rng, counters);
    W.leaf = 0;
  }
  if (active && !ended && W.cur != kWalkDone && !walk_at_node(W))
    ended = walk_other<kAnyHit, kCount, kFullShading>(S, W, stack, rng, counters);
  const bool done = active && (ended || (W.cur == kWalkDone && W.leaf == 0));
  if (done) walk_check_end(S, W);
  return done;
}

template <bool kCount = false, bool kFullShading = true>
__device__ __forceinline__ bool trace_closest(const SceneView& S, F3 o, F3 d, float tmin,
    float tmax, uint32_t& rng, Hit& hit, TraversalCounters* counters = nullptr) {
  bool found;
  traverse<false, kCount, kFullShading>(S, o, d, tmin, tmax, rng, hit, found, counters);
  return found;
}

template <bool kCount = false, bool kFullShading = true>
__device__ __forceinline__ float trace_shadow(const SceneView& S, F3 o, F3 d, float tmin,
    float tmax, TraversalCounters* counters = nullptr) {
  uint32_t rng = 0;
  Hit hit;
  bool found;
  return traverse<true, kCount, kFullShading>(S, o, d, tmin, tmax, rng, hit, found, counters);
}

}  // namespace lotus
