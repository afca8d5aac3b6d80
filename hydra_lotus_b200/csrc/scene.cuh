// SPDX-License-Identifier: Apache-2.0
// The GPU scene as the kernels read it, and software ray traversal.
//
// B200 has no RT cores, so the reference's ray queries (TraceRayInline over
// a driver-built TLAS/BLAS, backend/vulkan/shaders/common/scene.slang:
// 424-460 in hydra-lotus) become a two-level BVH walk:
//   - one BLAS per geometry in object space, one TLAS over the instances'
//     world boxes; all BLAS nodes share one pool and all triangles another;
//   - 64-byte nodes holding both children's boxes by axis, so one node is
//     four 16-byte loads and tests both children;
//   - triangles stored in leaf order as three float4 corners (48 bytes),
//     the original primitive index in the first corner's w;
//   - instance records split by use: a traversal record (object-from-world
//     rows, BLAS root, flags) and a shading record (world-from-object rows,
//     material, light-table offset, normals).
// Triangles are intersected with the watertight test of Woop, Benthin and
// Wald (JCGT 2013) in object space. Equal hit distances resolve to the
// smaller (instance, primitive), so the closest hit does not depend on the
// traversal order.
#pragma once

#include "common.cuh"

namespace lotus {

// Child encoding: >= 0 an interior node index in the same pool; < 0 a leaf
// whose first primitive is ~child (a triangle-pool index in a BLAS, an
// instance in the TLAS) with `count` primitives.
constexpr int32_t kEmptyChild = 0x7FFFFFFF;
constexpr int32_t kExitInstance = 0x7FFFFFFE;
constexpr int kStackSize = 96;
// A walk that visits more nodes than this ends early: only a corrupt BVH
// could need it, and the bound keeps such a walk from spinning.
constexpr uint32_t kMaxTraversalSteps = 1u << 18;

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

// lotus_material as five float4.
struct alignas(16) MaterialRecord {
  float4 base_roughness;       // base colour, roughness
  float4 emission_metallic;    // emission, metallic
  float4 specular_ior;         // specular colour, ior
  float4 transmission;         // transmission colour, transmission
  float4 coverage;             // opacity, threshold, flags (bits), reserved
};
static_assert(sizeof(MaterialRecord) == 80, "material record is 80 bytes");

// A light-table entry (GpuLightRecord, gpu_scene.hpp:120-126).
struct alignas(16) LightRecord {
  float pdf;
  float threshold;
  uint32_t alias;
  uint32_t instance;
};

struct SceneView {
  const BvhNode* __restrict__ tlas;
  const BvhNode* __restrict__ blas;
  const float4* __restrict__ tris;          // 3 per leaf-ordered triangle
  const InstanceTraversal* __restrict__ inst_trav;
  const InstanceShading* __restrict__ inst_shade;
  const MaterialRecord* __restrict__ materials;
  const float* __restrict__ normals;        // 9 floats per original triangle
  const LightRecord* __restrict__ lights;
  const float4* __restrict__ light_verts;   // 3 world corners per light entry
  const float4* __restrict__ light_radiance;// emission * coverage per light entry
  const float4* __restrict__ env_texels;
  const float* __restrict__ env_floats;     // density, marginal, conditional
  uint32_t instance_count;
  uint32_t light_count;
  uint32_t env_bound;
  uint32_t env_width, env_height, env_columns, env_rows;
  float env_selection;
  float env_scale[3];
  float env_frame[9];       // rows of environment_from_world
  float env_constant[3];
};

struct Hit {
  uint32_t instance;
  uint32_t tri;        // leaf-ordered triangle-pool index
  uint32_t primitive;  // the geometry's own triangle index
  float b1, b2;
  float t;
};

// Coverage (scene.slang:393-406) of a material's constant opacity.
__device__ __forceinline__ float material_coverage(const MaterialRecord& m) {
  const float opacity = m.coverage.x;
  const float threshold = m.coverage.y;
  if (threshold > 0.0f) return opacity >= threshold ? 1.0f : 0.0f;
  return opacity;
}

__device__ __forceinline__ float instance_coverage(const SceneView& S, uint32_t instance) {
  return material_coverage(S.materials[S.inst_trav[instance].material]);
}

__device__ __forceinline__ F3 safe_inverse(F3 d) {
  auto inv = [](float x) {
    return 1.0f / (fabsf(x) > 1e-30f ? x : (x < 0.0f ? -1e-30f : 1e-30f));
  };
  return V(inv(d.x), inv(d.y), inv(d.z));
}

struct WatertightRay {
  F3 org;
  int kx, ky, kz;
  float sx, sy, sz;
};

__device__ __forceinline__ WatertightRay prepare_ray(F3 org, F3 dir) {
  WatertightRay w;
  w.org = org;
  const float ax = fabsf(dir.x), ay = fabsf(dir.y), az = fabsf(dir.z);
  w.kz = ax > ay ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
  w.kx = w.kz == 2 ? 0 : w.kz + 1;
  w.ky = w.kx == 2 ? 0 : w.kx + 1;
  if (component(dir, w.kz) < 0.0f) {
    const int s = w.kx;
    w.kx = w.ky;
    w.ky = s;
  }
  const float dz = component(dir, w.kz);
  w.sx = component(dir, w.kx) / dz;
  w.sy = component(dir, w.ky) / dz;
  w.sz = 1.0f / dz;
  return w;
}

__device__ __forceinline__ bool intersect_triangle(const WatertightRay& r, F3 v0, F3 v1, F3 v2,
    float& t, float& b1, float& b2) {
  const F3 A = v0 - r.org, B = v1 - r.org, C = v2 - r.org;
  const float Akz = component(A, r.kz), Bkz = component(B, r.kz), Ckz = component(C, r.kz);
  const float Ax = component(A, r.kx) - r.sx * Akz;
  const float Ay = component(A, r.ky) - r.sy * Akz;
  const float Bx = component(B, r.kx) - r.sx * Bkz;
  const float By = component(B, r.ky) - r.sy * Bkz;
  const float Cx = component(C, r.kx) - r.sx * Ckz;
  const float Cy = component(C, r.ky) - r.sy * Ckz;
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

// Slab test of a node's two children against [tmin, tmax]. The far
// distance gets a relative margin of 2^-18 (the clamp to tmax included), so
// a box is never culled where the triangle test, whose distances carry
// their own rounding, could still accept a hit: hits are decided by
// triangle tests alone, whatever the BVH's shape.
__device__ __forceinline__ void test_children(const BvhNode& n, F3 o, F3 inv, float tmin,
    float tmax, bool& hit0, bool& hit1, float& near0, float& near1) {
  const float x0 = (n.x.x - o.x) * inv.x, x1 = (n.x.y - o.x) * inv.x;
  const float y0 = (n.y.x - o.y) * inv.y, y1 = (n.y.y - o.y) * inv.y;
  const float z0 = (n.z.x - o.z) * inv.z, z1 = (n.z.y - o.z) * inv.z;
  const float X0 = (n.x.z - o.x) * inv.x, X1 = (n.x.w - o.x) * inv.x;
  const float Y0 = (n.y.z - o.y) * inv.y, Y1 = (n.y.w - o.y) * inv.y;
  const float Z0 = (n.z.z - o.z) * inv.z, Z1 = (n.z.w - o.z) * inv.z;
  const float tn0 = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), tmin));
  const float tf0 = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), tmax));
  const float tn1 = fmaxf(fmaxf(fminf(X0, X1), fminf(Y0, Y1)), fmaxf(fminf(Z0, Z1), tmin));
  const float tf1 = fminf(fminf(fmaxf(X0, X1), fmaxf(Y0, Y1)), fminf(fmaxf(Z0, Z1), tmax));
  hit0 = tn0 <= tf0 + fabsf(tf0) * 3.8146973e-6f && n.c.x != kEmptyChild;
  hit1 = tn1 <= tf1 + fabsf(tf1) * 3.8146973e-6f && n.c.y != kEmptyChild;
  near0 = tn0;
  near1 = tn1;
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

// Walks the two-level BVH. kAnyHit: the shadow query of ShadowTransmittance
// (scene.slang:445-460), returning the transmittance; otherwise the closest
// accepted hit of Trace (scene.slang:424-439), whose coverage tests draw
// from `rng`.
template <bool kAnyHit, bool kCount>
__device__ __forceinline__ float traverse(const SceneView& S, F3 origin, F3 direction, float tmin,
    float tmax, uint32_t& rng, Hit& hit, bool& found, TraversalCounters* counters = nullptr) {
  found = false;
  float best = tmax;
  float transmittance = 1.0f;
  uint32_t best_instance = 0, best_prim = 0;
  int32_t stack[kStackSize];
  int sp = 0;
  F3 o = origin, d = direction;
  F3 inv = safe_inverse(d);
  WatertightRay w;
  const BvhNode* __restrict__ pool = S.tlas;
  uint32_t instance = 0;
  bool instance_opaque = true;
  int32_t cur = S.instance_count ? 0 : kEmptyChild;
  int32_t count = 0;
  if (cur == kEmptyChild) return kAnyHit ? 1.0f : 0.0f;
  for (uint32_t steps = 0; steps < kMaxTraversalSteps; ++steps) {
    if (cur >= 0 && cur != kExitInstance) {
      const BvhNode n = pool[cur];
      if (kCount) ++counters->nodes;
      bool h0, h1;
      float t0, t1;
      test_children(n, o, inv, tmin, best, h0, h1, t0, t1);
      if (h0 && h1) {
        const bool first0 = t0 <= t1;
        const int32_t near_c = first0 ? n.c.x : n.c.y;
        const int32_t far_c = first0 ? n.c.y : n.c.x;
        const int32_t near_n = first0 ? n.c.z : n.c.w;
        const int32_t far_n = first0 ? n.c.w : n.c.z;
        if (far_c < 0) {
          // Leaves go on the stack with their count in the next slot.
          if (sp + 2 <= kStackSize) {
            stack[sp++] = far_n;
            stack[sp++] = far_c;
          }
        } else if (sp < kStackSize) {
          stack[sp++] = far_c;
        }
        cur = near_c;
        count = near_n;
        continue;
      }
      if (h0 || h1) {
        cur = h0 ? n.c.x : n.c.y;
        count = h0 ? n.c.z : n.c.w;
        continue;
      }
    } else if (cur == kExitInstance) {
      // Back in world space.
      pool = S.tlas;
      o = origin;
      d = direction;
      inv = safe_inverse(d);
    } else if (pool == S.tlas) {
      // A TLAS leaf: enter each instance in turn. The TLAS leaves hold one
      // instance, so `count` is 1.
      instance = (uint32_t)(~cur);
      if (kCount) ++counters->instances;
      const InstanceTraversal rec = S.inst_trav[instance];
      if (rec.blas_root != (uint32_t)kEmptyChild && sp < kStackSize) {
        stack[sp++] = kExitInstance;
        o = row_point(rec.inv, origin);
        d = row_vector(rec.inv, direction);
        inv = safe_inverse(d);
        w = prepare_ray(o, d);
        instance_opaque = (rec.flags & kInstanceOpaque) != 0;
        pool = S.blas;
        cur = (int32_t)rec.blas_root;
        count = 0;
        continue;
      }
    } else {
      // BLAS leaf: `count` triangles from ~cur.
      const uint32_t first = (uint32_t)(~cur);
      for (int32_t k = 0; k < count; ++k) {
        const float4* tv = S.tris + 3 * (size_t)(first + k);
        const float4 a = tv[0], b = tv[1], c = tv[2];
        if (kCount) ++counters->triangles;
        float t, b1, b2;
        if (!intersect_triangle(w, V(a), V(b), V(c), t, b1, b2)) continue;
        if (!(t >= tmin) || !(t <= best)) continue;
        const uint32_t prim = __float_as_uint(a.w);
        if (kAnyHit) {
          const float coverage = instance_opaque ? 1.0f : instance_coverage(S, instance);
          if (coverage >= 1.0f) {
            found = true;
            return 0.0f;
          }
          if (coverage > 0.0f) transmittance *= 1.0f - coverage;
        } else {
          if (found && t == best &&
              (instance > best_instance || (instance == best_instance && prim >= best_prim)))
            continue;
          if (!instance_opaque) {
            const float coverage = instance_coverage(S, instance);
            if (coverage <= 0.0f) continue;
            if (coverage < 1.0f && !(next_random(rng) < coverage)) continue;
          }
          found = true;
          best = t;
          best_instance = instance;
          best_prim = prim;
          hit.instance = instance;
          hit.tri = first + k;
          hit.primitive = prim;
          hit.b1 = b1;
          hit.b2 = b2;
          hit.t = t;
        }
      }
    }
    if (sp == 0) break;
    cur = stack[--sp];
    if (cur < 0) count = stack[--sp];
  }
  return kAnyHit ? transmittance : 0.0f;
}

template <bool kCount = false>
__device__ __forceinline__ bool trace_closest(const SceneView& S, F3 o, F3 d, float tmin,
    float tmax, uint32_t& rng, Hit& hit, TraversalCounters* counters = nullptr) {
  bool found;
  traverse<false, kCount>(S, o, d, tmin, tmax, rng, hit, found, counters);
  return found;
}

template <bool kCount = false>
__device__ __forceinline__ float trace_shadow(const SceneView& S, F3 o, F3 d, float tmin,
    float tmax, TraversalCounters* counters = nullptr) {
  uint32_t rng = 0;
  Hit hit;
  bool found;
  return traverse<true, kCount>(S, o, d, tmin, tmax, rng, hit, found, counters);
}

}  // namespace lotus
