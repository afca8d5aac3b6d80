// SPDX-License-Identifier: Apache-2.0
// Temporal records and helpers: the primary-surface products, history
// validity, radiance history and the ReSTIR DI reservoirs, with the byte
// layouts of the reference's records (include/lotus/temporal.hpp:193-235,
// include/lotus/vulkan_backend.hpp:152-178 and the RestirSurface of
// backend/vulkan/shaders/common/restir.slang:44-60 in hydra-lotus), so that
// products read back from the device are the reference's types.
#pragma once

#include "transport.cuh"

namespace lotus {

struct alignas(16) TemporalPixel {
  float4 normal_depth;   // unit world geometric normal facing the camera, view depth
  float4 motion_depth;   // backward motion (px), expected previous depth, valid projection
  unsigned long long instance_id;
  unsigned long long material_id;
  uint32_t flags;        // 1 hit, 2 rigid correspondence, 4 unchanged material
  uint32_t albedo;       // unorm8 RGB
  uint32_t shading_normal;  // octahedral snorm16
  uint32_t reserved;
};
static_assert(sizeof(TemporalPixel) == 64, "TemporalPixel is 64 bytes");

struct alignas(16) ValidityPixel {
  uint32_t valid;
  uint32_t rejection;
  uint32_t previous_index;
  uint32_t reserved;
};

struct alignas(16) RadiancePixel {
  float4 color;
  uint32_t sample_count;
  float first_moment;
  float second_moment;
  float variance;
};
static_assert(sizeof(RadiancePixel) == 32, "RadiancePixel is 32 bytes");

struct Reservoir {
  uint32_t sample;
  float weight_sum;
  float selected_target;
  uint32_t candidate_count;
};

struct alignas(16) RestirPixel {
  Reservoir reservoir;
  float uv[2];
  float proposal;
  uint32_t flags;   // 1: camera surface, 2: invalid arithmetic
  float4 contribution;
};
static_assert(sizeof(RestirPixel) == 48, "RestirPixel is 48 bytes");

struct alignas(16) RestirReuse {
  RestirPixel pixel;
  float normalization;
  uint32_t supporting_candidates;
  uint32_t previous_index;
  uint32_t age;
};
static_assert(sizeof(RestirReuse) == 64, "RestirReuse is 64 bytes");

struct alignas(16) RestirSurface {
  float4 origin;          // offset origin, view depth
  float4 normal;          // w: dielectric_f90
  float4 shading_normal;  // w: transmission, negated for a thin wall
  float4 outgoing;        // w: eta, negated when smooth
  float4 base_alpha;
  float4 dielectric_metallic;
  float4 fresnel;
  float4 model;
  float4 extension;
  unsigned long long instance_id;
  unsigned long long material_id;
};
static_assert(sizeof(RestirSurface) == 160, "RestirSurface is 160 bytes");

// Per instance: the stable identities a temporal stream compares and the
// preceding frame's transform (TemporalInstanceRecord).
struct alignas(16) TemporalInstance {
  float4 previous[3];  // previous world_from_object rows
  unsigned long long instance_id;
  unsigned long long material_id;
  uint32_t flags;      // 2: rigid correspondence, 4: unchanged material
  uint32_t reserved[3];
};
static_assert(sizeof(TemporalInstance) == 80, "TemporalInstance is 80 bytes");

// Pixel (px, py) of a one-thread-per-pixel launch's thread `index`.
__device__ __forceinline__ bool pixel_of(uint32_t index, uint32_t width, uint32_t height,
    uint32_t& px, uint32_t& py) {
  if (index >= width * height) return false;
  px = index % width;
  py = index / width;
  return true;
}

__device__ __forceinline__ bool finite4(float4 v) {
  return isfinite(v.x) && isfinite(v.y) && isfinite(v.z) && isfinite(v.w);
}

constexpr uint32_t kNoReservoirSample = 0xFFFFFFFFu;
constexpr uint32_t kNoFilterGuide = 0xFFFFFFFFu;

// The temporal frame's constants (TemporalConstants,
// backend/vulkan/shaders/common/temporal.slang:10-24) and ReSTIR's.
struct TemporalConst {
  float current_view[16];
  float previous_view[16];
  float previous_world_to_clip[16];  // Vulkan clip
  float previous_display[4];
  uint32_t previous_data[4];
  float validation[4];    // absolute depth, relative depth, normal cosine, motion px
  uint32_t history;       // preceding frame available
  uint32_t width, height;
  uint32_t accumulate;
  uint32_t fresh_samples;
  uint32_t history_cap;
  uint32_t filter_iterations;
  uint32_t moments_half;  // the accumulation stores its moments at half precision
  uint32_t restir_candidates;
  uint32_t restir_history;     // temporal reuse reads the preceding reservoirs
  uint32_t restir_max_history;
  uint32_t restir_spatial;
  uint32_t restir_temporal;
  uint32_t restir_radius;
  uint32_t restir_neighbours;  // 0: four axis neighbours; else disk neighbours
  uint32_t restir_proposal;
  uint32_t sample_index;
  uint32_t max_bounces;
};

// mul(m, float4(p, w)) of a column-major 4x4 matrix.
__device__ __forceinline__ float4 mul4(const float* m, float x, float y, float z, float w) {
  return make_float4(m[0] * x + m[4] * y + m[8] * z + m[12] * w,
                     m[1] * x + m[5] * y + m[9] * z + m[13] * w,
                     m[2] * x + m[6] * y + m[10] * z + m[14] * w,
                     m[3] * x + m[7] * y + m[11] * z + m[15] * w);
}

// Rec. 709 luminance (TemporalLuminance).
__device__ __forceinline__ float luminance(float r, float g, float b) {
  return 0.2126f * r + 0.7152f * g + 0.0722f * b;
}

__device__ __forceinline__ uint32_t pack_albedo(F3 c) {
  const uint32_t x = (uint32_t)rintf(saturate(c.x) * 255.0f);
  const uint32_t y = (uint32_t)rintf(saturate(c.y) * 255.0f);
  const uint32_t z = (uint32_t)rintf(saturate(c.z) * 255.0f);
  return x | (y << 8) | (z << 16);
}

__device__ __forceinline__ F3 unpack_albedo(uint32_t a) {
  return V(float(a & 0xffu) / 255.0f, float((a >> 8) & 0xffu) / 255.0f, float((a >> 16) & 0xffu) / 255.0f);
}

// Octahedral snorm16 normal (temporal.slang:111-126).
__device__ __forceinline__ uint32_t pack_normal(F3 n) {
  const float s = fabsf(n.x) + fabsf(n.y) + fabsf(n.z);
  float ex = n.x / s, ey = n.y / s;
  if (n.z < 0.0f) {
    const float ox = (1.0f - fabsf(ey)) * (ex >= 0.0f ? 1.0f : -1.0f);
    const float oy = (1.0f - fabsf(ex)) * (ey >= 0.0f ? 1.0f : -1.0f);
    ex = ox;
    ey = oy;
  }
  const int qx = (int)rintf(fminf(fmaxf(ex, -1.0f), 1.0f) * 32767.0f);
  const int qy = (int)rintf(fminf(fmaxf(ey, -1.0f), 1.0f) * 32767.0f);
  return ((uint32_t)qx & 0xffffu) | ((uint32_t)qy << 16);
}

__device__ __forceinline__ F3 unpack_normal(uint32_t v) {
  const float ex = fmaxf(float((int)(v << 16) >> 16) / 32767.0f, -1.0f);
  const float ey = fmaxf(float((int)v >> 16) / 32767.0f, -1.0f);
  F3 n = V(ex, ey, 1.0f - fabsf(ex) - fabsf(ey));
  const float fold = fmaxf(-n.z, 0.0f);
  n.x += n.x >= 0.0f ? -fold : fold;
  n.y += n.y >= 0.0f ? -fold : fold;
  return n / sqrtf(dot(n, n));
}

__device__ __forceinline__ F3 demodulate(F3 c, uint32_t albedo) {
  const F3 a = unpack_albedo(albedo);
  return V(a.x > 0.0f ? c.x / a.x : c.x, a.y > 0.0f ? c.y / a.y : c.y, a.z > 0.0f ? c.z / a.z : c.z);
}

__device__ __forceinline__ F3 remodulate(F3 c, uint32_t albedo) {
  const F3 a = unpack_albedo(albedo);
  return V(a.x > 0.0f ? c.x * a.x : c.x, a.y > 0.0f ? c.y * a.y : c.y, a.z > 0.0f ? c.z * a.z : c.z);
}

// ---------------------------------------------------------------------------
// Reservoir arithmetic in float (reservoir.slang:23-103).

__device__ __forceinline__ Reservoir empty_reservoir() {
  Reservoir r;
  r.sample = kNoReservoirSample;
  r.weight_sum = 0.0f;
  r.selected_target = 0.0f;
  r.candidate_count = 0;
  return r;
}

__device__ __forceinline__ bool stream_candidate(Reservoir& r, uint32_t sample, float target,
    float proposal, float random, bool& selected) {
  selected = false;
  const bool valid_zero = r.weight_sum == 0.0f && r.sample == kNoReservoirSample && r.selected_target == 0.0f;
  const bool valid_positive = r.weight_sum > 0.0f && r.sample != kNoReservoirSample &&
      r.selected_target > 0.0f && r.candidate_count != 0;
  if (!isfinite(r.weight_sum) || !isfinite(r.selected_target) || !(valid_zero || valid_positive) ||
      !isfinite(target) || target < 0.0f || !isfinite(proposal) || proposal <= 0.0f ||
      !isfinite(random) || random < 0.0f || random >= 1.0f ||
      (target > 0.0f && sample == kNoReservoirSample) || r.candidate_count == 0xFFFFFFFFu)
    return false;
  const float weight = target / proposal;
  const float sum = r.weight_sum + weight;
  if (!isfinite(weight) || !isfinite(sum) || (target > 0.0f && weight == 0.0f)) return false;
  selected = weight > 0.0f && (r.weight_sum == 0.0f || random < weight / sum);
  r.weight_sum = sum;
  ++r.candidate_count;
  if (selected) {
    r.sample = sample;
    r.selected_target = target;
  }
  return true;
}

__device__ __forceinline__ float reservoir_normalization(const Reservoir& r) {
  return r.weight_sum > 0.0f ? (r.weight_sum / float(r.candidate_count)) / r.selected_target : 0.0f;
}

__device__ __forceinline__ bool merge_reevaluated(Reservoir& d, const Reservoir& s,
    float normalization, float target, uint32_t cap, float random, bool& selected) {
  selected = false;
  const uint32_t count = min(s.candidate_count, cap);
  const bool zero = s.weight_sum == 0.0f && s.sample == kNoReservoirSample && s.selected_target == 0.0f &&
      normalization == 0.0f && target == 0.0f;
  const bool positive = s.weight_sum > 0.0f && s.selected_target > 0.0f && s.sample != kNoReservoirSample &&
      s.candidate_count != 0 && normalization > 0.0f;
  const bool valid_destination = d.weight_sum == 0.0f
      ? d.sample == kNoReservoirSample && d.selected_target == 0.0f
      : d.weight_sum > 0.0f && d.selected_target > 0.0f && d.sample != kNoReservoirSample &&
          d.candidate_count != 0;
  if (!valid_destination || !isfinite(d.weight_sum) || !isfinite(d.selected_target) ||
      !isfinite(s.weight_sum) || !isfinite(s.selected_target) || !(zero || positive) ||
      !isfinite(normalization) || !isfinite(target) || target < 0.0f || cap == 0 ||
      !isfinite(random) || random < 0.0f || random >= 1.0f || count > 0xFFFFFFFFu - d.candidate_count)
    return false;
  const float weight = (target * normalization) * float(count);
  const float sum = d.weight_sum + weight;
  if (!isfinite(weight) || !isfinite(sum) || (target > 0.0f && weight == 0.0f)) return false;
  selected = weight > 0.0f && (d.weight_sum == 0.0f || random < weight / sum);
  d.weight_sum = sum;
  d.candidate_count += count;
  if (selected) {
    d.sample = s.sample;
    d.selected_target = target;
  }
  return true;
}

__device__ __forceinline__ float reuse_normalization(const Reservoir& r, uint32_t supporting) {
  return r.weight_sum > 0.0f ? (r.weight_sum / float(supporting)) / r.selected_target : 0.0f;
}

// ---------------------------------------------------------------------------
// The light-table domain reservoirs sample (scene.slang:915-967).

// ChooseReservoirLight: a light-table slot from two unit numbers under the
// proposal (0 power, 1 uniform, 2 equal mixture).
__device__ __forceinline__ uint32_t choose_reservoir_light(const SceneView& S, uint32_t proposal,
    float ux, float uy) {
  const uint32_t column = min((uint32_t)(ux * float(S.light_count)), S.light_count - 1);
  if (proposal == 1) return column;
  if (proposal == 2) {
    if (uy < 0.5f) return column;
    uy = (uy - 0.5f) * 2.0f;
  }
  const LightRecord record = S.lights[column];
  return uy < record.threshold ? column : record.alias;
}

__device__ __forceinline__ float reservoir_proposal_pdf(const SceneView& S, uint32_t proposal,
    uint32_t index) {
  const float power = S.lights[index].pdf;
  const float uniform = 1.0f / float(S.light_count);
  if (proposal == 1) return uniform;
  if (proposal == 2) return 0.5f * (power + uniform);
  return power;
}

// ReconstructReservoirLight: the candidate (ux, uy) of light-table slot
// `index`. Emissive triangles, rects and disks by area, the environment and
// distant lights by their receiver-independent maps; a sphere light's
// candidates are points uniform over its whole area, back-facing ones
// carrying nothing. kAnalytic = false leaves out the analytic lights' code,
// kFullShading = false the texture lookups', for scenes without them.
template <bool kAnalytic = true, bool kFullShading = true>
__device__ __forceinline__ LightSample reconstruct_reservoir_light(const SceneView& S,
    uint32_t index, float ux, float uy, F3 origin) {
  const LightRecord chosen = S.lights[index];
  if (chosen.instance == kEnvironmentLight) return sample_environment(S, chosen.pdf, ux, uy);
  if (!kAnalytic || (chosen.instance & kAnalyticLight) == 0)
    return sample_triangle<kFullShading>(S, index, chosen.pdf, ux, uy, origin);
  const AnalyticLight& light = S.analytic[chosen.instance & ~kAnalyticLight];
  if (light.shape != kSphereLight) return sample_analytic(light, chosen.pdf, ux, uy, origin);
  const float z = 1.0f - 2.0f * ux;
  const float radius_xy = sqrtf(fmaxf(0.0f, 1.0f - z * z));
  const float phi = 2.0f * kPi * uy;
  float sn, cs;
  lsincos(phi, sn, cs);
  const F3 normal = V(radius_xy * cs, radius_xy * sn, z);
  const F3 toward = V(light.position) + light.position.w * normal - origin;
  const float distance2 = dot(toward, toward);
  if (!(distance2 > 0.0f)) return no_light();
  LightSample s = no_light();
  s.distance = sqrtf(distance2);
  s.direction = toward / s.distance;
  const float cosine = -dot(normal, s.direction);
  if (!(cosine > 0.0f)) return no_light();
  s.radiance = V(light.radiance);
  s.pdf = chosen.pdf * distance2 / (cosine * 4.0f * kPi * light.position.w * light.position.w);
  return s;
}

// ReservoirPartitionPdf (scene.slang:973-983): SampleLight's density for
// the reservoir sample's direction, which for a sphere light is its cone's.
__device__ __forceinline__ float reservoir_partition_pdf(const SceneView& S, uint32_t index,
    const LightSample& ls, F3 origin) {
  const LightRecord chosen = S.lights[index];
  if ((chosen.instance & kAnalyticLight) != 0 && chosen.instance != kEnvironmentLight) {
    const AnalyticLight& light = S.analytic[chosen.instance & ~kAnalyticLight];
    if (light.shape == kSphereLight) {
      const F3 offset = V(light.position) - origin;
      return chosen.pdf * sphere_cone_pdf(light.position.w * light.position.w / dot(offset, offset));
    }
  }
  return ls.pdf;
}

}  // namespace lotus
