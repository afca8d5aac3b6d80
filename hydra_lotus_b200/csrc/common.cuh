// SPDX-License-Identifier: Apache-2.0
// Device vector math, the random sequence and shading frames
// (backend/vulkan/shaders/sampling/sampling.slang in hydra-lotus).
//
// The library is built with --fmad=false: every multiply and add in the
// transport rounds separately, in the order written here, which is the
// order of the reference's Slang source.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "lmath.cuh"

namespace lotus {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kFloatMax = 3.402823466e+38f;
constexpr uint32_t kNoLights = 0xFFFFFFFFu;
constexpr uint32_t kEnvironmentLight = 0xFFFFFFFFu;
// An analytic light's table entry has this bit in `instance`; the other
// bits index the analytic records (gpu_scene.hpp:128-131). The shapes
// (gpu_scene.hpp:136-142; a distant light of angle 0 is a parallel light),
// and the crossing hierarchy's child encoding (gpu_scene.hpp:168-172).
constexpr uint32_t kAnalyticLight = 0x80000000u;
constexpr uint32_t kSphereLight = 0, kRectLight = 1, kDiskLight = 2, kDistantLight = 3, kParallelLight = 4;
constexpr uint32_t kLightLeaf = 0x80000000u;
constexpr uint32_t kNoLightChild = 0xFFFFFFFFu;
// The crossing hierarchy's depth is at most ceil(log2(lights)); the host
// refuses more lights than this stack holds levels for.
constexpr uint32_t kLightStackSize = 32;

struct F3 {
  float x, y, z;
};

__host__ __device__ __forceinline__ F3 V(float x, float y, float z) { return F3{x, y, z}; }
__host__ __device__ __forceinline__ F3 V(float s) { return F3{s, s, s}; }
__host__ __device__ __forceinline__ F3 V(float4 a) { return F3{a.x, a.y, a.z}; }
__host__ __device__ __forceinline__ F3 operator+(F3 a, F3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ F3 operator-(F3 a, F3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ F3 operator-(F3 a) { return V(-a.x, -a.y, -a.z); }
__host__ __device__ __forceinline__ F3 operator*(F3 a, F3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
__host__ __device__ __forceinline__ F3 operator*(F3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ F3 operator*(float s, F3 a) { return V(s * a.x, s * a.y, s * a.z); }
__host__ __device__ __forceinline__ F3 operator/(F3 a, float s) { return V(a.x / s, a.y / s, a.z / s); }
__host__ __device__ __forceinline__ float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ F3 cross(F3 a, F3 b) {
  return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// 1/sqrt with both steps correctly rounded, as the oracle computes it.
__device__ __forceinline__ float rsqrt_rn(float x) { return 1.0f / sqrtf(x); }
__device__ __forceinline__ F3 normalize(F3 a) { return a * rsqrt_rn(dot(a, a)); }
__device__ __forceinline__ float length(F3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ float saturate(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }
__device__ __forceinline__ float max_component(F3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
__device__ __forceinline__ bool is_finite(F3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
__device__ __forceinline__ float component(F3 a, int axis) { return axis == 0 ? a.x : (axis == 1 ? a.y : a.z); }
__device__ __forceinline__ float4 F4(F3 a, float w) { return make_float4(a.x, a.y, a.z, w); }

// The PCG RXS-M-XS permutation as a hash (Jarzynski and Olano, "Hash
// Functions for GPU Rendering", JCGT 2020), as PcgHash, SeedRandom and
// NextRandom use it (sampling.slang:9-25).
__device__ __forceinline__ uint32_t pcg_hash(uint32_t value) {
  const uint32_t state = value * 747796405u + 2891336453u;
  const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}

__device__ __forceinline__ uint32_t seed_random(uint32_t pixel_index, uint32_t sample_index) {
  return pcg_hash(pixel_index ^ pcg_hash(sample_index));
}

// The next 24-bit uniform number in [0, 1).
__device__ __forceinline__ float next_random(uint32_t& state) {
  state = state * 747796405u + 2891336453u;
  const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return float(((word >> 22u) ^ word) >> 8u) * (1.0f / 16777216.0f);
}

// Orthonormal frame about a unit normal (Duff et al., JCGT 2017), as
// MakeShadingFrame builds it (sampling.slang:45-55).
struct Frame {
  F3 t, b, n;
  __device__ __forceinline__ F3 to_local(F3 d) const { return V(dot(d, t), dot(d, b), dot(d, n)); }
  __device__ __forceinline__ F3 to_world(F3 d) const { return d.x * t + d.y * b + d.z * n; }
};

__device__ __forceinline__ Frame make_frame(F3 n) {
  const float sign = n.z >= 0.0f ? 1.0f : -1.0f;
  const float a = -1.0f / (sign + n.z);
  const float b = n.x * n.y * a;
  Frame f;
  f.t = V(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
  f.b = V(b, sign + n.y * n.y * a, -n.y);
  f.n = n;
  return f;
}

// Veach's power heuristic in ratio form (sampling.slang:67-76).
__device__ __forceinline__ float power_heuristic(float chosen, float other) {
  if (!(chosen > 0.0f)) return 0.0f;
  if (isinf(chosen)) return isinf(other) ? 0.5f : 1.0f;
  const float ratio = other / chosen;
  return 1.0f / (1.0f + ratio * ratio);
}

// Cosine-weighted hemisphere about +z (sampling.slang:79-84).
__device__ __forceinline__ F3 sample_cosine_hemisphere(float ux, float uy) {
  const float radius = sqrtf(ux);
  const float phi = 2.0f * kPi * uy;
  float s, c;
  lsincos(phi, s, c);
  return V(radius * c, radius * s, sqrtf(fmaxf(0.0f, 1.0f - ux)));
}

// Waechter and Binder's self-intersection offset (Ray Tracing Gems 2019),
// as OffsetRayOrigin applies it (scene.slang:1454-1469).
__device__ __forceinline__ float offset_axis(float p, float n) {
  const float kOrigin = 1.0f / 32.0f;
  const float kFloatScale = 1.0f / 65536.0f;
  const float kIntScale = 256.0f;
  const int offset = (int)(kIntScale * n);
  const float moved = __int_as_float(__float_as_int(p) + (p < 0.0f ? -offset : offset));
  return fabsf(p) < kOrigin ? p + kFloatScale * n : moved;
}

__device__ __forceinline__ F3 offset_ray_origin(F3 p, F3 n) {
  return V(offset_axis(p.x, n.x), offset_axis(p.y, n.y), offset_axis(p.z, n.z));
}

}  // namespace lotus
