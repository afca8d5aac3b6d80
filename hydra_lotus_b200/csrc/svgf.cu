// SPDX-License-Identifier: Apache-2.0
// SVGF's temporal accumulation, variance estimate, a-trous iterations and
// composite (backend/vulkan/shaders/common/temporal.slang:229-475 in
// hydra-lotus). One thread per pixel; every pass is a separate launch, so
// each reads only what the preceding one finished writing. Checked against
// the reference's own CPU code (temporal.cpp) within its published GPU
// tolerances. Built without fused multiply-adds all the same: fused, the
// variance estimate's and the filter's edge-stopping and neighbour tests
// (depth steps and luminance differences against thresholds) decided
// differently from the CPU code at one to three pixels of a 64x64 frame,
// each then far outside the tolerance.
#include <cuda_fp16.h>

#include "../../include/lotus_cuda.h"
#include "temporal_passes.cuh"

namespace lotus {
namespace {

constexpr int kBlock = 128;

// ---------------------------------------------------------------------------
// SVGF.

// A luminance moment rounded to half precision (round to nearest even),
// saturating at the largest finite half, 65504 (a NaN stays a NaN, so the
// next frame drops the history as the FP32 mode does).
__device__ __forceinline__ float half_moment(float m) {
  return __half2float(__float2half_rn(m > 65504.0f ? 65504.0f : m));
}

// The FP16 moment mode keeps the first moment and the central second
// moment, m2 - m1^2, each at half precision: the raw second moment in half
// precision would lose the variance to cancellation wherever it is small
// beside m1^2 (a half's relative step of 2^-11 of m2 exceeds it), and the
// variance is what SVGF's edge-stopping weighs. The second moment a pass
// reads is then the central one plus the stored first moment squared.
__device__ __forceinline__ float second_moment(const TemporalConst& tc, const RadiancePixel& r) {
  return tc.moments_half ? r.second_moment + r.first_moment * r.first_moment : r.second_moment;
}

// AccumulateTemporalRadiance (temporal.slang:229-267), without history
// rectification: the count-capped blend of the fresh batch and the
// reprojected history, and its illumination luminance moments.
__global__ void __launch_bounds__(kBlock) k_svgf_accumulate(const TemporalConst* __restrict__ tcp,
    const float4* __restrict__ batch, const TemporalPixel* __restrict__ surface,
    const ValidityPixel* __restrict__ validity, const RadiancePixel* __restrict__ old,
    RadiancePixel* __restrict__ out) {
  const TemporalConst& tc = *tcp;
  uint32_t px, py;
  if (!pixel_of(blockIdx.x * blockDim.x + threadIdx.x, tc.width, tc.height, px, py)) return;
  const uint32_t index = py * tc.width + px;
  RadiancePixel o = {};
  o.color = batch[index];
  const uint32_t cap = tc.history_cap;
  const TemporalPixel s = surface[index];
  if ((s.flags & 1u) != 0) {
    o.sample_count = min(tc.fresh_samples, cap);
    const F3 d = demodulate(V(o.color), s.albedo);
    const float l = luminance(d.x, d.y, d.z);
    float m1 = l, m2 = l * l;
    const ValidityPixel v = validity[index];
    if (v.valid != 0) {
      const RadiancePixel h = old[v.previous_index];
      const uint32_t kept = min(h.sample_count, cap - o.sample_count);
      if (kept != 0 && finite4(h.color) && isfinite(h.first_moment) && isfinite(h.second_moment)) {
        const uint32_t count = kept + o.sample_count;
        const float blend = float(kept) / float(count);
        o.color.x += (h.color.x - o.color.x) * blend;
        o.color.y += (h.color.y - o.color.y) * blend;
        o.color.z += (h.color.z - o.color.z) * blend;
        o.color.w += (h.color.w - o.color.w) * blend;
        m1 += (h.first_moment - m1) * blend;
        m2 += (second_moment(tc, h) - m2) * blend;
        o.sample_count = count;
      }
    }
    if (tc.moments_half) {
      m1 = half_moment(m1);
      m2 = half_moment(fmaxf(m2 - m1 * m1, 0.0f));
    }
    o.first_moment = m1;
    o.second_moment = m2;
  }
  out[index] = o;
}

__device__ __forceinline__ bool variance_neighbour(const TemporalConst& tc, int qx, int qy,
    unsigned long long instance_id, const RadiancePixel* radiance, const TemporalPixel* surface) {
  if (qx < 0 || qy < 0 || qx >= (int)tc.width || qy >= (int)tc.height) return false;
  const uint32_t i = (uint32_t)qy * tc.width + (uint32_t)qx;
  return radiance[i].sample_count != 0 && surface[i].instance_id == instance_id;
}

__device__ __forceinline__ float variance_depth_step(const TemporalConst& tc, int ax, int ay, int bx,
    int by, float depth, unsigned long long id, const RadiancePixel* radiance, const TemporalPixel* surface) {
  float step = -1.0f;
  if (variance_neighbour(tc, ax, ay, id, radiance, surface))
    step = fabsf(depth - surface[(uint32_t)ay * tc.width + (uint32_t)ax].normal_depth.w);
  if (variance_neighbour(tc, bx, by, id, radiance, surface)) {
    const float other = fabsf(depth - surface[(uint32_t)by * tc.width + (uint32_t)bx].normal_depth.w);
    step = step < 0.0f ? other : fminf(step, other);
  }
  return fmaxf(step, 0.0f);
}

// EstimateTemporalVariance (temporal.slang:313-370): temporal variance from
// four or more batches, else the 7x7 edge-aware moments estimate; with a
// filter, also iteration 0's input and the guides.
__global__ void __launch_bounds__(kBlock) k_svgf_variance(const TemporalConst* __restrict__ tcp,
    const TemporalPixel* __restrict__ surface, RadiancePixel* __restrict__ radiance,
    float4* __restrict__ filter) {
  const TemporalConst& tc = *tcp;
  uint32_t px, py;
  if (!pixel_of(blockIdx.x * blockDim.x + threadIdx.x, tc.width, tc.height, px, py)) return;
  const int x = (int)px, y = (int)py;
  const uint32_t index = py * tc.width + px;
  const RadiancePixel center = radiance[index];
  float variance = 0.0f;
  const float batches = float(center.sample_count) / float(min(tc.fresh_samples, tc.history_cap));
  if (center.sample_count != 0) {
    if (batches >= 4.0f) {
      variance = fmaxf(0.0f, second_moment(tc, center) - center.first_moment * center.first_moment);
    } else {
      const TemporalPixel s = surface[index];
      const float depth = s.normal_depth.w;
      const float phi = fmaxf(variance_depth_step(tc, x - 1, y, x + 1, y, depth, s.instance_id, radiance, surface) +
          variance_depth_step(tc, x, y - 1, x, y + 1, depth, s.instance_id, radiance, surface), 1.0e-8f) * 3.0f;
      float weight_sum = 0.0f, s1 = 0.0f, s2 = 0.0f;
      for (int dy = -3; dy <= 3; ++dy) {
        for (int dx = -3; dx <= 3; ++dx) {
          const int qx = x + dx, qy = y + dy;
          if (!variance_neighbour(tc, qx, qy, s.instance_id, radiance, surface)) continue;
          const uint32_t qi = (uint32_t)qy * tc.width + (uint32_t)qx;
          const float4 n = surface[qi].normal_depth;
          const RadiancePixel nb = radiance[qi];
          const float distance = sqrtf(float(dx * dx + dy * dy));
          const float wz = dx == 0 && dy == 0 ? 0.0f : fabsf(depth - n.w) / (phi * distance);
          const float wn = powf(saturate(dot(V(s.normal_depth), V(n))), 128.0f);
          const float wl = fabsf(center.first_moment - nb.first_moment) / 10.0f;
          const float w = expf(-(wl + wz)) * wn;
          s1 += w * nb.first_moment;
          s2 += w * second_moment(tc, nb);
          weight_sum += w;
        }
      }
      const float m1 = s1 / fmaxf(weight_sum, 1.0e-6f), m2 = s2 / fmaxf(weight_sum, 1.0e-6f);
      variance = fmaxf(0.0f, m2 - m1 * m1) * (4.0f / batches);
    }
  }
  radiance[index].variance = variance;
  if (tc.filter_iterations == 0) return;
  const uint32_t pixels = tc.width * tc.height;
  float4 input = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  uint4 guide = make_uint4(0u, 0u, kNoFilterGuide, 0u);
  if (center.sample_count != 0) {
    const TemporalPixel s = surface[index];
    const F3 d = demodulate(V(center.color), s.albedo);
    input = F4(d, variance / batches);
    guide = make_uint4((uint32_t)s.instance_id, (uint32_t)(s.instance_id >> 32),
        __float_as_uint(s.normal_depth.w), s.shading_normal);
  }
  filter[index] = input;
  filter[2 * pixels + index] = make_float4(__uint_as_float(guide.x), __uint_as_float(guide.y),
      __uint_as_float(guide.z), __uint_as_float(guide.w));
  // The guide's shading normal unpacked once per frame (the a-trous taps
  // read it instead of unpacking it 25 times per iteration).
  filter[3 * pixels + index] =
      center.sample_count != 0 ? F4(unpack_normal(guide.w), 0.0f) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

__device__ __forceinline__ uint4 filter_guide(const float4* filter, uint32_t pixels, uint32_t i) {
  const float4 g = filter[2 * pixels + i];
  return make_uint4(__float_as_uint(g.x), __float_as_uint(g.y), __float_as_uint(g.z), __float_as_uint(g.w));
}

__device__ __forceinline__ bool filter_neighbour(const TemporalConst& tc, const float4* filter, int qx,
    int qy, uint32_t ix, uint32_t iy, uint4& guide) {
  guide = make_uint4(0u, 0u, kNoFilterGuide, 0u);
  if (qx < 0 || qy < 0 || qx >= (int)tc.width || qy >= (int)tc.height) return false;
  guide = filter_guide(filter, tc.width * tc.height, (uint32_t)qy * tc.width + (uint32_t)qx);
  return guide.z != kNoFilterGuide && guide.x == ix && guide.y == iy;
}

__device__ __forceinline__ float filter_depth_step(const TemporalConst& tc, const float4* filter, int ax,
    int ay, int bx, int by, float depth, uint32_t ix, uint32_t iy) {
  float step = -1.0f;
  uint4 g;
  if (filter_neighbour(tc, filter, ax, ay, ix, iy, g)) step = fabsf(depth - __uint_as_float(g.z));
  if (filter_neighbour(tc, filter, bx, by, ix, iy, g)) {
    const float other = fabsf(depth - __uint_as_float(g.z));
    step = step < 0.0f ? other : fminf(step, other);
  }
  return fmaxf(step, 0.0f);
}

// FilterIteration (temporal.slang:405-457).
__device__ __forceinline__ float4 filter_iteration(const TemporalConst& tc, const float4* __restrict__ filter,
    int x, int y, uint32_t iteration) {
  const uint32_t pixels = tc.width * tc.height;
  const uint32_t index = (uint32_t)y * tc.width + (uint32_t)x;
  const uint4 center = filter_guide(filter, pixels, index);
  if (center.z == kNoFilterGuide) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const float4* in = filter + (size_t)(iteration & 1u) * pixels;
  uint4 g;
  float gaussian = 0.0f, gaussian_weight = 0.0f;
#pragma unroll
  for (int dy = -1; dy <= 1; ++dy) {
#pragma unroll
    for (int dx = -1; dx <= 1; ++dx) {
      const int qx = x + dx, qy = y + dy;
      if (!filter_neighbour(tc, filter, qx, qy, center.x, center.y, g)) continue;
      const float k = (dx == 0 ? 0.5f : 0.25f) * (dy == 0 ? 0.5f : 0.25f);
      gaussian += k * in[(uint32_t)qy * tc.width + (uint32_t)qx].w;
      gaussian_weight += k;
    }
  }
  const float phi_l = 4.0f * sqrtf(fmaxf(gaussian / gaussian_weight, 0.0f) + 1.0e-10f);
  const float depth = __uint_as_float(center.z);
  const float phi_z = fmaxf(filter_depth_step(tc, filter, x - 1, y, x + 1, y, depth, center.x, center.y) +
      filter_depth_step(tc, filter, x, y - 1, x, y + 1, depth, center.x, center.y), 1.0e-8f);
  const F3 normal = V(filter[3 * (size_t)pixels + index]);
  const float4 cv = in[index];
  const float lum = luminance(cv.x, cv.y, cv.z);
  const int step = 1 << iteration;
  const float kernel[3] = {0.375f, 0.25f, 0.0625f};
  // The edge-stopping divisions as products: 1 / phi_l, and 1 / (phi_z *
  // distance) for the five tap distances (squared 1, 2, 4, 5, 8 steps).
  const float inv_phi_l = 1.0f / phi_l;
  float inv_depth[9];
#pragma unroll
  for (int d2 = 1; d2 <= 8; ++d2) inv_depth[d2] = 1.0f / (phi_z * (float(step) * sqrtf(float(d2))));
  float sx = 0.0f, sy = 0.0f, sz = 0.0f, var = 0.0f, weight_sum = 0.0f;
#pragma unroll
  for (int ty = -2; ty <= 2; ++ty) {
#pragma unroll
    for (int tx = -2; tx <= 2; ++tx) {
      const int qx = x + tx * step, qy = y + ty * step;
      if (!filter_neighbour(tc, filter, qx, qy, center.x, center.y, g)) continue;
      const float4 value = in[(uint32_t)qy * tc.width + (uint32_t)qx];
      float w = kernel[abs(tx)] * kernel[abs(ty)];
      if (tx != 0 || ty != 0) {
        const F3 other = V(filter[3 * (size_t)pixels + (uint32_t)qy * tc.width + (uint32_t)qx]);
        const float facing = saturate(dot(normal, other));
        // A neighbour facing away weighs 0 (pow(0, 128)): its tap adds nothing.
        if (facing == 0.0f) continue;
        const float wz = fabsf(depth - __uint_as_float(g.z)) * inv_depth[tx * tx + ty * ty];
        const float wl = fabsf(lum - luminance(value.x, value.y, value.z)) * inv_phi_l;
        const float wn = powf(facing, 128.0f);
        w = w * expf(-(wl + wz)) * wn;
      }
      sx += w * value.x;
      sy += w * value.y;
      sz += w * value.z;
      var += w * w * value.w;
      weight_sum += w;
    }
  }
  return make_float4(sx / weight_sum, sy / weight_sum, sz / weight_sum, var / (weight_sum * weight_sum));
}

// One a-trous iteration (FilterTemporalRadiance, temporal.slang:459-464),
// or, for the last, the composite (temporal.slang:468-475) into the colour.
__global__ void __launch_bounds__(kBlock) k_svgf_filter(const TemporalConst* __restrict__ tcp,
    float4* __restrict__ filter, uint32_t iteration, uint32_t composite,
    const RadiancePixel* __restrict__ radiance, const TemporalPixel* __restrict__ surface,
    float4* __restrict__ color) {
  const TemporalConst& tc = *tcp;
  uint32_t px, py;
  if (!pixel_of(blockIdx.x * blockDim.x + threadIdx.x, tc.width, tc.height, px, py)) return;
  const uint32_t index = py * tc.width + px;
  const uint32_t pixels = tc.width * tc.height;
  if (!composite) {
    filter[(size_t)((iteration + 1) & 1u) * pixels + index] = filter_iteration(tc, filter, (int)px, (int)py, iteration);
    return;
  }
  const RadiancePixel r = radiance[index];
  if (r.sample_count == 0) {
    color[index] = r.color;
    return;
  }
  const float4 v = filter_iteration(tc, filter, (int)px, (int)py, iteration);
  color[index] = F4(remodulate(V(v), surface[index].albedo), r.color.w);
}

// The radiance history's colour as the frame's colour (no filter).
__global__ void k_copy_radiance_color(const TemporalConst* __restrict__ tcp,
    const RadiancePixel* __restrict__ radiance, float4* __restrict__ color) {
  const TemporalConst& tc = *tcp;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < tc.width * tc.height) color[i] = radiance[i].color;
}

inline uint32_t grid(uint32_t n) { return (n + kBlock - 1) / kBlock; }

}  // namespace

void launch_svgf(const TemporalConst* tc, const TemporalConst& host_tc, const float4* batch,
    const TemporalPixel* surface, const ValidityPixel* validity, const RadiancePixel* old,
    RadiancePixel* radiance, float4* filter, float4* color, uint32_t pixels, cudaStream_t s) {
  k_svgf_accumulate<<<grid(pixels), kBlock, 0, s>>>(tc, batch, surface, validity, old, radiance);
  k_svgf_variance<<<grid(pixels), kBlock, 0, s>>>(tc, surface, radiance, filter);
  if (host_tc.filter_iterations == 0) {
    k_copy_radiance_color<<<grid(pixels), kBlock, 0, s>>>(tc, radiance, color);
    return;
  }
  for (uint32_t i = 0; i < host_tc.filter_iterations; ++i)
    k_svgf_filter<<<grid(pixels), kBlock, 0, s>>>(tc, filter, i, i + 1 == host_tc.filter_iterations ? 1u : 0u,
        radiance, surface, color);
}

}  // namespace lotus
