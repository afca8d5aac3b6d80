// SPDX-License-Identifier: Apache-2.0
// The reference path tracer as one megakernel, and the wavefront path
// tracer as camera, shade, shadow and extend kernels over compacted queues
// (backend/vulkan/shaders/path_trace.slang, wavefront/wavefront.slang and
// common/transport.slang in hydra-lotus).
//
// Both integrators run the same scattering code and draw each path's random
// numbers in the same order, so a pixel and sample index select the same
// path in either. The wavefront shade kernel defers next event estimation's
// shadow ray to the shadow kernel, which adds the light to the path's
// radiance before the next extension reads it, so the radiance sums run in
// the reference's order.
#include <algorithm>
#include <mutex>
#include <type_traits>
#include <utility>
#include <vector>

#include "../../include/lotus_cuda.h"
#include "integrator.cuh"
#include "temporal.cuh"

namespace lotus {

namespace {

constexpr int kBlock = 128;

// Pixels in warp tiles of 8 x 4 for coherent camera rays.
__device__ __forceinline__ bool tile_pixel(uint32_t index, const uint32_t* rect, uint32_t& px,
    uint32_t& py) {
  const uint32_t tiles_x = (rect[2] + 7) / 8;
  const uint32_t tile = index >> 5, lane = index & 31u;
  const uint32_t tx = tile % tiles_x, ty = tile / tiles_x;
  const uint32_t x = tx * 8 + (lane & 7u), y = ty * 4 + (lane >> 3);
  px = rect[0] + x;
  py = rect[1] + y;
  return x < rect[2] && y < rect[3];
}

__host__ __device__ __forceinline__ uint32_t tile_threads(const uint32_t* rect) {
  return ((rect[2] + 7) / 8) * ((rect[3] + 3) / 4) * 32;
}

// Appends `pred` lanes of the (converged) warp to a queue: one atomic per
// warp, slots in lane order.
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool pred) {
  const unsigned mask = __ballot_sync(0xFFFFFFFFu, pred);
  const unsigned lane = threadIdx.x & 31u;
  uint32_t base = 0;
  if (mask) {
    const int leader = __ffs(mask) - 1;
    if ((int)lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
  }
  return base + (uint32_t)__popc(mask & ((1u << lane) - 1u));
}

// The reordering key's grid: the box of the TLAS root's children (the
// scene's box), kSortAxisBits cells per axis.
struct SortGrid {
  float lo[3];
  float scale[3];
};

__device__ __forceinline__ SortGrid sort_grid(const SceneView& S) {
  SortGrid g;
  float hi[3];
  for (int a = 0; a < 3; ++a) {
    g.lo[a] = 3.0e38f;
    hi[a] = -3.0e38f;
    g.scale[a] = 0.0f;
  }
  if (S.tlas == nullptr || S.instance_count == 0) return g;
  const Bvh4Node& r = S.tlas[0];
  const int child[4] = {r.child.x, r.child.y, r.child.z, r.child.w};
  const float lx[4] = {r.lo_x.x, r.lo_x.y, r.lo_x.z, r.lo_x.w}, hx[4] = {r.hi_x.x, r.hi_x.y, r.hi_x.z, r.hi_x.w};
  const float ly[4] = {r.lo_y.x, r.lo_y.y, r.lo_y.z, r.lo_y.w}, hy[4] = {r.hi_y.x, r.hi_y.y, r.hi_y.z, r.hi_y.w};
  const float lz[4] = {r.lo_z.x, r.lo_z.y, r.lo_z.z, r.lo_z.w}, hz[4] = {r.hi_z.x, r.hi_z.y, r.hi_z.z, r.hi_z.w};
  for (int i = 0; i < 4; ++i) {
    if (child[i] == kEmptyChild) continue;
    g.lo[0] = fminf(g.lo[0], lx[i]); hi[0] = fmaxf(hi[0], hx[i]);
    g.lo[1] = fminf(g.lo[1], ly[i]); hi[1] = fmaxf(hi[1], hy[i]);
    g.lo[2] = fminf(g.lo[2], lz[i]); hi[2] = fmaxf(hi[2], hz[i]);
  }
  for (int a = 0; a < 3; ++a)
    g.scale[a] = hi[a] > g.lo[a] ? (float)(1u << kSortAxisBits) / (hi[a] - g.lo[a]) : 0.0f;
  return g;
}

// Every third bit from bit 0 for the low ten bits of v.
__device__ __forceinline__ uint32_t spread_bits3(uint32_t v) {
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

// A batch's keys lead with the scene, and its cells are coarser: six bits
// of scene (LOTUS_BATCH_MAX_SCENES), three per axis, then the octant.
constexpr uint32_t kBatchSortAxisBits = 3;
static_assert(LOTUS_BATCH_MAX_SCENES <= (1u << (3 * (kSortAxisBits - kBatchSortAxisBits))),
    "a batch's scene index fits above its cells");

template <uint32_t kAxisBits>
__device__ __forceinline__ uint32_t sort_key(const SortGrid& g, const F3& o, const F3& d) {
  const float p[3] = {o.x, o.y, o.z};
  constexpr uint32_t top = (1u << kAxisBits) - 1u;
  // The grid's scale is for kSortAxisBits cells per axis.
  constexpr float coarse = 1.0f / (float)(1u << (kSortAxisBits - kAxisBits));
  uint32_t cell[3];
  for (int a = 0; a < 3; ++a) {
    const float v = (p[a] - g.lo[a]) * g.scale[a] * coarse;
    cell[a] = v > 0.0f ? (v < (float)top ? (uint32_t)v : top) : 0u;
  }
  const uint32_t morton = spread_bits3(cell[0]) | (spread_bits3(cell[1]) << 1) | (spread_bits3(cell[2]) << 2);
  const uint32_t octant = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
  return (morton << 3) | octant;
}

__device__ __forceinline__ void warp_add64(unsigned long long* counter, uint32_t value) {
  unsigned long long v = value;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
  if ((threadIdx.x & 31u) == 0 && v) atomicAdd(counter, v);
}

// The scene of a batch that owns path slot `slot` (binary search over the
// scenes' slot ranges).
__device__ __forceinline__ uint32_t table_scene(const SceneTable& B, uint32_t slot) {
  uint32_t lo = 0, hi = B.count;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (B.slot_base[mid] <= slot) lo = mid;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ bool frame_rect_contains(const FrameConst& f, uint32_t px, uint32_t py) {
  return px >= f.rect[0] && py >= f.rect[1] && px < f.rect[0] + f.rect[2] && py < f.rect[1] + f.rect[3];
}

// The light a pending shadow ray carries once its transmittance is known.
__device__ __forceinline__ F3 shadow_contribution(F3 fl, float weight, float pdf,
    float transmittance) {
  const F3 c = fl * (transmittance * weight / pdf);
  return is_finite(c) ? c : V(0.0f);
}

// ParallelLights (transport.slang:139-146): under BSDF sampling, the
// parallel lights, which no sampled direction finds, each through its own
// shadow ray traced here, as ShadowedLight carries a delta light. Not
// inlined: the shading kernels hold none of the walk's registers for it.
template <bool kFullShading>
__device__ __noinline__ F3 parallel_lights(const SceneView& S, F3 position, F3 normal, const SurfaceHit& sh,
    const Frame& basis, F3 wo, uint32_t& shadow_rays) {
  const F3 origin = offset_ray_origin(position, normal);
  F3 sum = V(0.0f);
  for (uint32_t index = 0; index < S.analytic_count; ++index) {
    const LightSample ls = parallel_light(S, index);
    F3 c = V(0.0f);
    if (ls.pdf > 0.0f && max_component(ls.radiance) > 0.0f && dot(ls.direction, normal) > 0.0f) {
      const F3 wi = basis.to_local(ls.direction);
      if (wi.z > 0.0f) {
        const F3 fv = surface_evaluate<kFullShading>(sh, wo, wi);
        if (max_component(fv) > 0.0f) {
          ++shadow_rays;
          const float tr = trace_shadow(S, origin, ls.direction, 0.0f, ls.distance);
          if (tr > 0.0f) c = shadow_contribution(fv * ls.radiance, 1.0f, ls.pdf, tr);
        }
      }
    }
    sum = sum + c;
  }
  return sum;
}

// Next event estimation's pending shadow ray.
struct ShadowRequest {
  uint32_t inline_shadow;  // shadow rays traced inside scatter (parallel lights)
  bool pending;
  F3 origin;
  F3 direction;
  float tmax;
  F3 fl;        // f * light radiance
  float weight; // MIS weight (1 for a delta light)
  float pdf;
  F3 throughput;
};

// ScatterPath (transport.slang:164-230): adds the hit's emission (weighed
// against light sampling) and that of the analytic lights the incoming ray
// crossed, applies Russian roulette, prepares next event estimation's
// shadow ray (under BSDF sampling, traces the parallel lights' own) and
// samples the BSDF. Returns whether the path continues along (new_o, new_d).
// kAnalytic: the scene may have analytic lights; kFullShading: texture
// lookups or glTF PBR materials (SceneView::full_shading). The
// instantiations without carry none of their code or registers.
template <bool kAnalytic, bool kFullShading>
__device__ __forceinline__ bool scatter(const SceneView& S, const FrameConst& f,
    uint32_t instance, uint32_t tri, float b1, float b2, F3 ray_o, F3 ray_d, uint32_t depth,
    F3& T, F3& R, float& last_pdf, uint32_t& flags, uint32_t& rng, F3& new_o, F3& new_d,
    ShadowRequest& req, uint32_t pixel_index, CacheRecord* features = nullptr, bool end_here = false) {
  req.pending = false;
  req.inline_shadow = 0;
  uint32_t primitive;
  const SurfaceHit sh = reconstruct_hit<kFullShading>(S, instance, tri, b1, b2, ray_d, &primitive);
  if (features) {
    // The radiance cache's description of this vertex, seen from the ray.
    const F3 albedo = sh.bsdf.transmission > 0.0f
        ? sh.base_color + sh.bsdf.transmission * (sh.bsdf.transmission_color - sh.base_color)
        : sh.base_color;
    features->pos_rough = F4(sh.position, sh.roughness);
    features->dir = F4(-ray_d, 0.0f);
    features->normal = F4(sh.shading_normal, 0.0f);
    features->albedo = F4(albedo, sh.metallic);
  }
  const bool weigh = f.sample_lights && (flags & kUnweightedLight) == 0;
  F3 emission = sh.emission;
  if (weigh && depth != 0 && max_component(emission) > 0.0f) {
    // EmissionWeight (transport.slang:150-158).
    const float area_pdf = emitter_pdf(S, instance, primitive, sh.area);
    float w = 1.0f;
    if (area_pdf > 0.0f) {
      const F3 toward = sh.position - ray_o;
      const float cosine = fabsf(dot(sh.normal, ray_d));
      w = power_heuristic(last_pdf, area_pdf * dot(toward, toward) / cosine);
    }
    emission = emission * w;
  }
  R = R + T * emission;
  // The analytic lights the ray crossed before the hit; camera rays do not
  // see them.
  if (kAnalytic && depth != 0 && S.analytic_count != 0)
    R = R + T * crossed_lights(S, ray_o, ray_d, dot(sh.position - ray_o, ray_d), false, weigh, last_pdf);
  if (depth >= f.max_bounces) return false;
  if (!end_here && depth >= kRouletteBounces) {
    const float survival = fminf(max_component(T), kMaxSurvival);
    if (next_random(rng) >= survival) return false;
    T = T / survival;
  }
  const Frame basis = make_frame(sh.shading_normal);
  const F3 wo = basis.to_local(-ray_d);
  if (f.restir_primary && depth == 0) {
    // InitialDirectLight (restir.slang:235-254): the final reservoir's
    // contribution, its visibility included, under the power-table/BSDF
    // partition weight.
    const RestirPixel sel = *reinterpret_cast<const RestirPixel*>(
        f.restir_final + (size_t)pixel_index * f.restir_stride);
    if ((sel.flags & 2u) == 0 && sel.reservoir.weight_sum > 0.0f && sel.reservoir.sample < S.light_count) {
      const F3 origin = offset_ray_origin(sh.position, sh.normal);
      const LightSample ls = reconstruct_reservoir_light<kAnalytic, kFullShading>(S, sel.reservoir.sample, sel.uv[0], sel.uv[1], origin);
      const F3 wi = basis.to_local(ls.direction);
      const float weight = ls.delta ? 1.0f
          : power_heuristic(kAnalytic ? reservoir_partition_pdf(S, sel.reservoir.sample, ls, origin) : ls.pdf,
                wi.z > 0.0f ? surface_pdf<kFullShading>(sh, wo, wi) : 0.0f);
      R = R + T * (V(sel.contribution) * weight);
    } else {
      R = R + T * V(0.0f);
    }
  } else if (f.sample_lights && S.light_count != 0) {
    // DirectLight and ShadowedLight up to the shadow ray
    // (transport.slang:82-135).
    const float u0 = next_random(rng);
    const float u1 = next_random(rng);
    const float u2 = next_random(rng);
    const float u3 = next_random(rng);
    const F3 origin = offset_ray_origin(sh.position, sh.normal);
    const LightSample ls = sample_light<kAnalytic, kFullShading>(S, u0, u1, u2, u3, origin);
    if (ls.pdf > 0.0f && max_component(ls.radiance) > 0.0f && dot(ls.direction, sh.normal) > 0.0f) {
      const F3 wi = basis.to_local(ls.direction);
      if (wi.z > 0.0f) {
        const F3 fv = surface_evaluate<kFullShading>(sh, wo, wi);
        if (max_component(fv) > 0.0f) {
          req.pending = true;
          req.origin = origin;
          req.direction = ls.direction;
          req.tmax = ls.distance;
          req.fl = fv * ls.radiance;
          req.weight = ls.delta ? 1.0f : power_heuristic(ls.pdf, surface_pdf<kFullShading>(sh, wo, wi));
          req.pdf = ls.pdf;
          req.throughput = T;
        }
      }
    }
  } else if (kAnalytic && !f.sample_lights && S.analytic_count != 0) {
    R = R + T * parallel_lights<kFullShading>(S, sh.position, sh.normal, sh, basis, wo, req.inline_shadow);
  }
  // A path that ends into the radiance cache stops after next event
  // estimation at its cache vertex: the cache stands for the light the
  // vertex scatters but its direct light, which the shadow ray brings.
  if (end_here) return false;
  F3 u;
  u.x = next_random(rng);
  u.y = next_random(rng);
  u.z = next_random(rng);
  BsdfSample s;
  if (!surface_sample<kFullShading>(sh, wo, u, s)) return false;
  const F3 wi = normalize(basis.to_world(s.wi));
  const float side = dot(wi, sh.normal);
  if (s.transmitted ? side >= 0.0f : side <= 0.0f) return false;
  T = T * s.weight;
  last_pdf = s.pdf;
  if (s.delta || s.transmitted)
    flags |= kUnweightedLight;
  else
    flags &= ~kUnweightedLight;
  new_o = offset_ray_origin(sh.position, s.transmitted ? -sh.normal : sh.normal);
  new_d = wi;
  return true;
}

// MissPath (transport.slang:235-247): an escaping continuation ray adds the
// environment's radiance, the image's weighed against light sampling, then
// that of the analytic lights it crossed.
template <bool kAnalytic>
__device__ __forceinline__ F3 miss_path(const SceneView& S, const FrameConst& f, F3 o, F3 d,
    uint32_t flags, float last_pdf, F3 T, F3 R) {
  const bool weigh = f.sample_lights && (flags & kUnweightedLight) == 0;
  F3 env = V(S.env_constant[0], S.env_constant[1], S.env_constant[2]);
  if (S.env_bound) env = env + environment_radiance(S, d, weigh, last_pdf);
  R = R + T * env;
  if (kAnalytic && S.analytic_count != 0) R = R + T * crossed_lights(S, o, d, kFloatMax, true, weigh, last_pdf);
  return R;
}

// The radiance pass's output (path_trace.slang:369-385) from the FP64
// accumulation: a pixel no sample has hit keeps the clear colour unless the
// environment image shows behind it.
__device__ __forceinline__ float4 resolve_pixel(const SceneView& S, const FrameConst& f,
    uint32_t px, uint32_t py, double4 sum) {
  // The samples in the accumulation once this wave's are added.
  const double count = (double)(f.accumulated + f.add_sample * max(f.wave, 1u));
  const bool env_shows = f.environment_background != 0 && S.env_bound != 0;
  if (sum.w == 0.0 && (!env_shows || count == 0.0))
    return make_float4(f.background[0], f.background[1], f.background[2], f.background[3]);
  double bg[4] = {f.background[0], f.background[1], f.background[2], f.background[3]};
  if (env_shows && sum.w < count) {
    F3 o, d;
    float tmax;
    camera_ray(f, (float(px) + 0.5f) * f.ndc[0] + f.ndc[2], (float(py) + 0.5f) * f.ndc[1] + f.ndc[3],
        o, d, tmax);
    const F3 e = environment_radiance(S, d, false, 0.0f);
    bg[0] = e.x;
    bg[1] = e.y;
    bg[2] = e.z;
    bg[3] = 1.0;
  }
  const double miss = count - sum.w;
  return make_float4((float)((sum.x + miss * bg[0]) / count), (float)((sum.y + miss * bg[1]) / count),
      (float)((sum.z + miss * bg[2]) / count), (float)((sum.w + miss * bg[3]) / count));
}

__device__ __forceinline__ double4 add4(double4 a, float4 s) {
  return make_double4(a.x + (double)s.x, a.y + (double)s.y, a.z + (double)s.z, a.w + (double)s.w);
}

// Resident blocks a SM of the per-thread path loops (the reference
// integrator, the tail kernel): four (at most 128 registers a thread)
// without analytic lights or full shading, else three (at most 168). The
// full-shading instantiations would otherwise take over 220 registers and
// keep a third of the warps resident.
constexpr int path_loop_blocks(bool analytic, bool full_shading) { return analytic || full_shading ? 3 : 4; }

// ---------------------------------------------------------------------------
// The reference integrator: one thread follows one camera path to its end
// (path_trace.slang:279-287, 353-385), then adds it to the pixel's FP64
// accumulation and writes the mean.
template <bool kCount, bool kAnalytic, bool kFullShading>
__global__ void __launch_bounds__(kBlock, path_loop_blocks(kAnalytic, kFullShading)) k_reference_pt(SceneView S,
    const FrameConst* __restrict__ fcp, double4* __restrict__ accum, float4* __restrict__ color,
    RayTotals* totals, VisitCounters* visits) {
  TraversalCounters vc[3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  const FrameConst& f = *fcp;
  const uint32_t rect[4] = {f.rect[0], f.rect[1], f.rect[2], f.rect[3]};
  uint32_t px, py;
  const uint32_t index = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = tile_pixel(index, rect, px, py);
  uint32_t n_camera = 0, n_extension = 0, n_shadow = 0;
  if (valid) {
    const uint32_t slot = py * f.width + px;
    double4 sum = f.accumulated != 0 ? accum[slot] : make_double4(0.0, 0.0, 0.0, 0.0);
    if (f.add_sample) {
      F3 o, d;
      float tmax;
      uint32_t rng;
      start_path(f, px, py, f.sample_index, o, d, tmax, rng);
      ++n_camera;
      Hit hit;
      if (trace_closest<kCount, kFullShading>(S, o, d, 0.0f, tmax, rng, hit, &vc[0])) {
        F3 T = V(1.0f), R = V(0.0f);
        float last_pdf = 0.0f;
        uint32_t flags = 0;
        for (uint32_t depth = 0;; ++depth) {
          F3 no, nd;
          ShadowRequest req;
          const bool cont = scatter<kAnalytic, kFullShading>(S, f, hit.instance, hit.tri, hit.b1, hit.b2, o, d, depth, T, R,
              last_pdf, flags, rng, no, nd, req, slot);
          n_shadow += req.inline_shadow;
          if (req.pending) {
            ++n_shadow;
            const float tr = trace_shadow<kCount, kFullShading>(S, req.origin, req.direction, 0.0f, req.tmax, &vc[2]);
            if (tr > 0.0f) R = R + req.throughput * shadow_contribution(req.fl, req.weight, req.pdf, tr);
          }
          if (!cont) break;
          o = no;
          d = nd;
          ++n_extension;
          if (!trace_closest<kCount, kFullShading>(S, o, d, 0.0f, kFloatMax, rng, hit, &vc[1])) {
            R = miss_path<kAnalytic>(S, f, o, d, flags, last_pdf, T, R);
            break;
          }
        }
        sum = add4(sum, make_float4(R.x, R.y, R.z, 1.0f));
      }
      accum[slot] = sum;
    }
    color[slot] = resolve_pixel(S, f, px, py, sum);
  }
  warp_add64(&totals->camera, n_camera);
  warp_add64(&totals->extension, n_extension);
  warp_add64(&totals->shadow, n_shadow);
  if (kCount) {
    const uint32_t rays[3] = {n_camera, n_extension, n_shadow};
    for (int k = 0; k < 3; ++k) {
      warp_add64(&visits->rays[k], rays[k]);
      warp_add64(&visits->nodes[k], vc[k].nodes);
      warp_add64(&visits->triangles[k], vc[k].triangles);
      warp_add64(&visits->instances[k], vc[k].instances);
    }
  }
}

// ---------------------------------------------------------------------------
// The wavefront integrator.

// Camera (wavefront.slang:206-225): starts each pixel's path and traces its
// camera ray; a hit is queued for shading at bounce 0.
// In a batch (kBatch) one thread per path slot of every scene, in each
// image's row order or in the table's warp tiles; otherwise 8x4 pixel
// tiles per warp.
template <bool kCount, bool kBatch, bool kFullShading>
__global__ void __launch_bounds__(kBlock) k_wf_camera(SceneView S,
    const FrameConst* __restrict__ fcp, PathState P, Queues Q, VisitCounters* visits, SceneTable B) {
  TraversalCounters vc = {0, 0, 0};
  const uint32_t index = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t px = 0, py = 0, slot = 0, scene = 0, wave_sample = 0;
  bool valid;
  if (kBatch) {
    slot = index;
    valid = index < B.total_slots;
    if (valid) {
      scene = table_scene(B, index);
      const FrameConst& fb = B.frames[scene];
      const uint32_t local = index - B.slot_base[scene];
      if (B.camera_tile) {
        const uint32_t k = B.camera_tile;
        const uint32_t tiles_x = fb.width >> k, tile = local >> 5, lane = local & 31u;
        px = ((tile % tiles_x) << k) + (lane & ((1u << k) - 1u));
        py = (tile / tiles_x) * (32u >> k) + (lane >> k);
        slot = B.slot_base[scene] + py * fb.width + px;
      } else {
        px = local % fb.width;
        py = local / fb.width;
      }
      valid = fb.add_sample && frame_rect_contains(fb, px, py);
    }
  } else {
    if (!fcp->add_sample) return;
    // The wave's samples one after another, each over the rect's tiles.
    const uint32_t rect[4] = {fcp->rect[0], fcp->rect[1], fcp->rect[2], fcp->rect[3]};
    const uint32_t per_sample = tile_threads(rect);
    wave_sample = index / per_sample;
    valid = wave_sample < max(fcp->wave, 1u) && tile_pixel(index - wave_sample * per_sample, rect, px, py);
    slot = wave_sample * fcp->wave_stride + py * fcp->width + px;
  }
  const FrameConst& f = kBatch ? B.frames[scene] : *fcp;
  const SceneView& SS = kBatch ? B.views[scene] : S;
  bool found = false;
  if (valid) {
    F3 o, d;
    float tmax;
    uint32_t rng;
    start_path(f, px, py, f.sample_index + wave_sample, o, d, tmax, rng);
    Hit hit;
    if (!kBatch && f.primary_hit != nullptr && wave_sample == 0 && f.sample_index == f.primary_sample) {
      // The same camera ray's hit, traced by a pass earlier in the frame.
      const uint4 ph = f.primary_hit[slot];
      found = ph.x != kNoPrimaryHit;
      hit.instance = ph.x;
      hit.tri = ph.y;
      hit.b1 = __uint_as_float(ph.z);
      hit.b2 = __uint_as_float(ph.w);
      rng = f.primary_rng[slot];
    } else {
      found = trace_closest<kCount, kFullShading>(SS, o, d, 0.0f, tmax, rng, hit, &vc);
    }
    if (found) {
      P.direction[slot] = F4(d, tmax);
      P.radiance[slot] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(rng));
      P.hit[slot] = make_uint4(hit.instance, hit.tri, __float_as_uint(hit.b1), __float_as_uint(hit.b2));
    } else {
      P.radiance[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
  }
  const uint32_t at = warp_append(&Q.counts[1], found);
  if (found) Q.hit[at] = slot;
  if (kCount) {
    warp_add64(&visits->rays[0], valid ? 1u : 0u);
    warp_add64(&visits->nodes[0], vc.nodes);
    warp_add64(&visits->triangles[0], vc.triangles);
    warp_add64(&visits->instances[0], vc.instances);
  }
}

// Shade (wavefront.slang:264-285) with next event estimation's shadow ray
// deferred to the shadow queue. With the radiance cache, the paths reaching
// the cache's vertex (bounce 1, the second vertex, unless configured
// otherwise) end into the cache there (a query of the
// cache records the vertex and the path's throughput), except the training
// paths, one in `stride` chosen per sample, which record the vertex, their
// throughput and radiance so far and carry on.
// kCacheVertex: the cache's vertex (bounce 1 with the cache enabled); the
// other instantiation carries none of the cache's code or registers.
// Compiled for six resident blocks per SM (80 registers): shading is
// latency-bound and gains more from occupancy than from registers. The
// full-shading instantiation (texture lookups, glTF PBR) at four (128
// registers): at 80 it spilled 350-550 bytes a thread.
constexpr int kShadeBlocksPerSm = 6;
template <bool kCacheVertex, bool kBatch, bool kAnalytic, bool kFullShading>
__global__ void __launch_bounds__(kBlock, kFullShading ? 4 : kShadeBlocksPerSm) k_wf_shade(SceneView S,
    const FrameConst* __restrict__ fcp, PathState P, Queues Q, uint32_t bounce, CacheQueues C, SceneTable B) {
  const uint32_t n = Q.counts[3 * bounce + 1];
  const bool cache_vertex = kCacheVertex && bounce < fcp->max_bounces;
  const bool keyed = Q.keys != nullptr;
  __shared__ SortGrid grids[kBatch ? LOTUS_BATCH_MAX_SCENES : 1];
  if (keyed) {
    if (kBatch) {
      for (uint32_t k = threadIdx.x; k < B.count; k += blockDim.x) grids[k] = sort_grid(B.views[k]);
    } else if (threadIdx.x == 0) {
      grids[0] = sort_grid(S);
    }
    __syncthreads();
  }
  // Grid-stride over the hit queue (the grid is sized to a few waves of
  // the SMs, not to the largest queue, so that the short queues of late
  // bounces cost little).
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const uint32_t index = base + threadIdx.x;
    const bool valid = index < n;
    bool cont = false, query = false, training = false;
    ShadowRequest req;
    req.pending = false;
    uint32_t slot = 0, key = 0;
    CacheRecord features;
    F3 T = V(1.0f), T_in = V(1.0f), R = V(0.0f);
    if (valid) {
      slot = Q.hit[index];
      const uint32_t scene = kBatch ? table_scene(B, slot) : 0u;
      const FrameConst& f = kBatch ? B.frames[scene] : *fcp;
      const SceneView& SS = kBatch ? B.views[scene] : S;
      const float4 dir = P.direction[slot];
      const float4 rad = P.radiance[slot];
      const uint4 h = P.hit[slot];
      float last_pdf = 0.0f;
      uint32_t flags = 0;
      F3 ro = V(0.0f);
      if (bounce != 0) {
        const float4 thr = P.throughput[slot];
        T = V(thr);
        last_pdf = thr.w;
        flags = last_pdf < 0.0f ? kUnweightedLight : 0u;
        if (f.sample_lights || (kAnalytic && SS.analytic_count != 0)) ro = V(P.origin[slot]);
      }
      T_in = T;
      R = V(rad);
      uint32_t rng = __float_as_uint(rad.w);
      if (cache_vertex)
        training = pcg_hash(slot ^ pcg_hash(f.sample_index ^ 0xC2B2AE35u)) % C.stride == 0u;
      F3 no, nd;
      cont = scatter<kAnalytic, kFullShading>(SS, f, h.x, h.y, __uint_as_float(h.z), __uint_as_float(h.w), ro, V(dir), bounce,
          T, R, last_pdf, flags, rng, no, nd, req, slot, cache_vertex ? &features : nullptr,
          cache_vertex && !training);
      query = cache_vertex && !training;
      if (cont) {
        if (keyed && kBatch)
          key = (scene << (3 * kBatchSortAxisBits + 3)) | sort_key<kBatchSortAxisBits>(grids[scene], no, nd);
        else if (keyed)
          key = sort_key<kSortAxisBits>(grids[0], no, nd);
        P.origin[slot] = F4(no, 0.0f);
        P.direction[slot] = F4(nd, kFloatMax);
        P.throughput[slot] = F4(T, (flags & kUnweightedLight) ? -1.0f : last_pdf);
        P.radiance[slot] = F4(R, __uint_as_float(rng));
      } else {
        P.radiance[slot] = F4(R, 1.0f);
      }
    }
    if (kCacheVertex) {
      const uint32_t q_at = warp_append(&C.counters[0], query);
      if (query && q_at < C.query_capacity) {
        C.queries[q_at] = features;
        C.query_slots[q_at] = slot;
        C.query_throughput[q_at] = F4(T_in, 0.0f);
        if (C.query_keys != nullptr) {
          const float p[3] = {features.pos_rough.x, features.pos_rough.y, features.pos_rough.z};
          constexpr uint32_t top = (1u << kQuerySortAxisBits) - 1u;
          uint32_t cell[3];
          for (int a = 0; a < 3; ++a) {
            const float v = (p[a] - C.grid_lo[a]) * C.grid_scale[a];
            cell[a] = v > 0.0f ? (v < (float)top ? (uint32_t)v : top) : 0u;
          }
          const uint32_t key = spread_bits3(cell[0]) | (spread_bits3(cell[1]) << 1) | (spread_bits3(cell[2]) << 2);
          C.query_keys[q_at] = key;
          const unsigned peers = __match_any_sync(__activemask(), key);
          if ((threadIdx.x & 31u) == (unsigned)(__ffs(peers) - 1))
            atomicAdd(&C.query_bins[key], (uint32_t)__popc(peers));
        }
      }
      const uint32_t t_at = warp_append(&C.counters[1], training);
      if (training && t_at < C.train_capacity) {
        C.train[t_at] = features;
        C.train_slots[t_at] = slot;
        C.train_throughput[t_at] = F4(T_in, 0.0f);
      }
    }
    const uint32_t ray_at = warp_append(&Q.counts[3 * (bounce + 1)], cont);
    if (cont) Q.ray[(bounce + 1) & 1][ray_at] = slot;
    if (keyed && cont) {
      // The key beside the ray, and one histogram increment per key held
      // by the warp's lanes.
      Q.keys[ray_at] = key;
      const unsigned peers = __match_any_sync(__activemask(), key);
      if ((threadIdx.x & 31u) == (unsigned)(__ffs(peers) - 1)) atomicAdd(&Q.bins[key], (uint32_t)__popc(peers));
    }
    const uint32_t sh_at = warp_append(&Q.counts[3 * bounce + 2], req.pending);
    if (req.pending) {
      Q.shadow.ray_o[sh_at] = F4(req.origin, req.tmax);
      Q.shadow.ray_d[sh_at] = F4(req.direction, req.weight);
      Q.shadow.fl[sh_at] = F4(req.fl, req.pdf);
      Q.shadow.thr[sh_at] = F4(req.throughput, __uint_as_float(slot));
    }
  }
}

// The training targets once the sample's paths have ended: the radiance a
// training path gathered after its cache vertex's emission and next event
// estimation, divided by its throughput on arrival there.
__global__ void k_cache_targets(CacheQueues C, PathState P) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t n = min(C.counters[1], C.train_capacity);
  if (i >= n) return;
  const float4 r = P.radiance[C.train_slots[i]];
  const float4 base = C.train_base[i];
  const float4 t = C.train_throughput[i];
  auto ratio = [](float a, float b) { return b > 0.0f ? fmaxf(a, 0.0f) / b : 0.0f; };
  float4 target = make_float4(ratio(r.x - base.x, t.x), ratio(r.y - base.y, t.y), ratio(r.z - base.z, t.z), 0.0f);
  if (!isfinite(target.x) || !isfinite(target.y) || !isfinite(target.z)) target = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  C.train_targets[i] = target;
}

// Each training path's radiance once its cache vertex's emission and shadow
// ray are in (after that bounce's shadow launch): what the cache's target
// leaves out.
__global__ void k_cache_base(CacheQueues C, PathState P) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t n = min(C.counters[1], C.train_capacity);
  if (i < n) C.train_base[i] = P.radiance[C.train_slots[i]];
}

constexpr unsigned kFullWarp = 0xFFFFFFFFu;
// Resident blocks per SM the persistent tracing kernels are compiled for:
// seven blocks of 128 (72 registers a thread; the extension walk spills a
// few words to L1) hide more of the node loads' latency than six at 80
// registers (sphere field, 1080p: extension kernels 2.30 -> 2.16 ms per
// sample together with the approximate slab reciprocal and the evict_last
// node loads).
constexpr int kTraceBlocksPerSm = 7;
constexpr uint32_t kDefaultRefillBelow = 24;

// The persistent kernels' ray fetch: when fewer than `refill_below` lanes
// of the warp hold a ray (and the queue is not exhausted), the idle lanes
// take the next queue entries with one atomic per warp. Returns the lane's
// queue index, or n when it got none.
__device__ __forceinline__ uint32_t warp_fetch(uint32_t* cursor, uint32_t n, bool active,
    uint32_t refill_below, bool& exhausted) {
  const unsigned act = __ballot_sync(kFullWarp, active);
  if (exhausted || (uint32_t)__popc(act) >= refill_below) return n;
  const unsigned need = ~act;
  const unsigned lane = threadIdx.x & 31u;
  uint32_t base = 0;
  if (lane == 0) base = atomicAdd(cursor, (uint32_t)__popc(need));
  base = __shfl_sync(kFullWarp, base, 0);
  exhausted = base + (uint32_t)__popc(need) >= n;
  if (active) return n;
  const uint32_t index = base + (uint32_t)__popc(need & ((1u << lane) - 1u));
  return index < n ? index : n;
}

// ShadowedLight's visibility (transport.slang:82-115) for the shadow queue,
// as a persistent kernel: each lane walks one shadow ray at a time and adds
// the light to the path's radiance when the ray arrives.
template <bool kCount, bool kBatch, bool kFullShading>
__global__ void __launch_bounds__(kBlock, kTraceBlocksPerSm) k_wf_shadow(SceneView S, PathState P, Queues Q,
    uint32_t bounce, uint32_t* __restrict__ fetch, uint32_t refill_below, VisitCounters* visits, SceneTable B) {
  const uint32_t n = Q.counts[3 * bounce + 2];
  TraversalCounters vc = {0, 0, 0};
  uint32_t rays = 0;
  Walk W;
  WalkStack stack;
  uint32_t rng = 0;
  uint32_t index = 0, scene = 0;
  bool active = false, exhausted = false;
  for (;;) {
    const uint32_t got = warp_fetch(fetch, n, active, refill_below, exhausted);
    if (got < n) {
      index = got;
      if (kBatch) scene = table_scene(B, __float_as_uint(Q.shadow.thr[index].w));
      const float4 ro = Q.shadow.ray_o[index];
      const float4 rd = Q.shadow.ray_d[index];
      walk_begin(kBatch ? B.views[scene] : S, W, V(ro), V(rd), 0.0f, ro.w);
      active = true;
      ++rays;
    }
    if (!__any_sync(kFullWarp, active)) break;
    if (walk_round<true, kCount, kFullShading>(kBatch ? B.views[scene] : S, W, stack, rng, active, &vc)) {
      active = false;
      const float tr = W.transmittance;
      if (tr > 0.0f) {
        const float4 rd = Q.shadow.ray_d[index];
        const float4 fl = Q.shadow.fl[index];
        const float4 thr = Q.shadow.thr[index];
        const uint32_t slot = __float_as_uint(thr.w);
        const F3 c = shadow_contribution(V(fl), rd.w, fl.w, tr);
        float4 rad = P.radiance[slot];
        const F3 R = V(rad) + V(thr) * c;
        rad.x = R.x;
        rad.y = R.y;
        rad.z = R.z;
        P.radiance[slot] = rad;
      }
    }
  }
  if (kCount) {
    warp_add64(&visits->rays[2], rays);
    warp_add64(&visits->nodes[2], vc.nodes);
    warp_add64(&visits->triangles[2], vc.triangles);
    warp_add64(&visits->instances[2], vc.instances);
  }
}

// The diagnostic outputs (CameraPass's surface pass, path_trace.slang:
// 67-98): the pixel centre's closest hit, traced with a fixed coverage
// sequence (sample 0), as its barycentric weights or a diagnostic of its
// surface; a miss leaves the pixel as it is (the clear colour).
__global__ void __launch_bounds__(kBlock) k_diagnostic(SceneView S, const FrameConst* __restrict__ fcp,
    uint32_t output, float4* __restrict__ color) {
  const FrameConst& f = *fcp;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= f.rect[2] * f.rect[3]) return;
  const uint32_t px = f.rect[0] + i % f.rect[2], py = f.rect[1] + i / f.rect[2];
  const uint32_t slot = py * f.width + px;
  uint32_t rng = seed_random(slot, 0);
  F3 o, d;
  float tmax;
  camera_ray(f, (float(px) + 0.5f) * f.ndc[0] + f.ndc[2], (float(py) + 0.5f) * f.ndc[1] + f.ndc[3], o, d, tmax);
  Hit hit;
  if (!trace_closest(S, o, d, 0.0f, tmax, rng, hit)) return;
  if (output == kOutputBarycentrics) {
    color[slot] = make_float4(1.0f - hit.b1 - hit.b2, hit.b1, hit.b2, 1.0f);
    return;
  }
  const SurfaceHit sh = reconstruct_hit(S, hit.instance, hit.tri, hit.b1, hit.b2, d);
  if (output == kOutputAlbedo)
    color[slot] = F4(sh.base_color, 1.0f);
  else if (output == kOutputRoughnessMetallic)
    color[slot] = make_float4(sh.roughness, sh.metallic, 0.0f, 1.0f);
  else
    color[slot] = F4(sh.shading_normal, 1.0f);
}

// The camera pass's depth (CameraPass, path_trace.slang:69-97): the pixel
// centre's closest hit, traced with the fixed coverage sequence of sample 0
// as the diagnostics are, as Vulkan window depth: the hit position through
// the frame's world-to-clip, z over w. A miss leaves the pixel's depth as
// it is (the clear depth, or the preceding frame's).
__global__ void __launch_bounds__(kBlock) k_depth(SceneView S, const FrameConst* __restrict__ fcp,
    float* __restrict__ depth) {
  const FrameConst& f = *fcp;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= f.rect[2] * f.rect[3]) return;
  const uint32_t px = f.rect[0] + i % f.rect[2], py = f.rect[1] + i / f.rect[2];
  const uint32_t slot = py * f.width + px;
  uint32_t rng = seed_random(slot, 0);
  F3 o, d;
  float tmax;
  camera_ray(f, (float(px) + 0.5f) * f.ndc[0] + f.ndc[2], (float(py) + 0.5f) * f.ndc[1] + f.ndc[3], o, d, tmax);
  Hit hit;
  if (!trace_closest(S, o, d, 0.0f, tmax, rng, hit)) return;
  const F3 p = o + d * hit.t;
  const float* m = f.world_to_clip;
  const float z = m[2] * p.x + m[6] * p.y + m[10] * p.z + m[14];
  const float w = m[3] * p.x + m[7] * p.y + m[11] * p.z + m[15];
  depth[slot] = z / w;
}

__global__ void k_fill_float(float* __restrict__ out, uint32_t n, float value) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = value;
}

// The ReSTIR passes' queued visibility rays (VisibilityQueue), as a
// persistent any-hit kernel that completes each ray's pixel record.
__global__ void __launch_bounds__(kBlock, kTraceBlocksPerSm) k_visibility(SceneView S, VisibilityQueue VQ,
    uint32_t pass, unsigned char* __restrict__ records, uint32_t stride, uint32_t positive,
    uint32_t refill_below) {
  const uint32_t n = VQ.counters[2 * pass];
  Walk W;
  WalkStack stack;
  uint32_t rng = 0, index = 0;
  bool active = false, exhausted = false;
  for (;;) {
    const uint32_t got = warp_fetch(&VQ.counters[2 * pass + 1], n, active, refill_below, exhausted);
    if (got < n) {
      index = got;
      const float4 o = VQ.origin[index];
      walk_begin(S, W, V(o), V(VQ.direction[index]), 0.0f, o.w);
      active = true;
    }
    if (!__any_sync(kFullWarp, active)) break;
    if (walk_round<true, false>(S, W, stack, rng, active, nullptr)) {
      active = false;
      const float visibility = W.transmittance;
      const uint32_t slot = VQ.slot[index];
      const float4 c = VQ.pending[slot];
      RestirPixel* p = reinterpret_cast<RestirPixel*>(records + (size_t)slot * stride);
      const F3 estimate = V(c) * (visibility * c.w);
      if (!isfinite(c.w) || (positive && c.w <= 0.0f) || !is_finite(estimate)) {
        p->flags |= 2u;
        atomicMin(&VQ.failed[pass], slot);
      } else
        p->contribution = F4(estimate, visibility);
    }
  }
}

// Intersect (wavefront.slang:230-262) as a persistent kernel: a hit is
// queued for shading; a miss ends the path with the environment. Each warp
// stages its hits in shared memory and appends them to the hit queue 32 at
// a time.
template <bool kCount, bool kBatch, bool kAnalytic, bool kFullShading>
__global__ void __launch_bounds__(kBlock, kTraceBlocksPerSm) k_wf_extend(SceneView S,
    const FrameConst* __restrict__ fcp, PathState P, Queues Q, const uint32_t* __restrict__ rays_in, uint32_t bounce,
    uint32_t* __restrict__ fetch, uint32_t refill_below, VisitCounters* visits, SceneTable B) {
  __shared__ uint32_t staged[kBlock / 32][64];
  const uint32_t n = Q.counts[3 * bounce];
  const unsigned lane = threadIdx.x & 31u;
  uint32_t* stage = staged[threadIdx.x >> 5];
  uint32_t* hits = &Q.counts[3 * bounce + 1];
  uint32_t staged_count = 0;
  TraversalCounters vc = {0, 0, 0};
  uint32_t rays = 0;
  Walk W;
  WalkStack stack;
  uint32_t rng = 0, rng0 = 0, slot = 0, scene = 0;
  bool active = false, exhausted = false;
  for (;;) {
    const uint32_t got = warp_fetch(fetch, n, active, refill_below, exhausted);
    if (got < n) {
      slot = rays_in[got];
      if (kBatch) scene = table_scene(B, slot);
      const float4 o = P.origin[slot];
      const float4 d = P.direction[slot];
      rng = rng0 = __float_as_uint(P.radiance[slot].w);
      walk_begin(kBatch ? B.views[scene] : S, W, V(o), V(d), o.w, d.w);
      active = true;
      ++rays;
    }
    if (!__any_sync(kFullWarp, active)) break;
    bool emit = false;
    const SceneView& SS = kBatch ? B.views[scene] : S;
    if (walk_round<false, kCount, kFullShading>(SS, W, stack, rng, active, &vc)) {
      active = false;
      if (W.found) {
        P.hit[slot] = make_uint4(W.best_instance, W.best_tri, __float_as_uint(W.b1), __float_as_uint(W.b2));
        if (rng != rng0) P.radiance[slot].w = __uint_as_float(rng);
        emit = true;
      } else {
        const float4 rad = P.radiance[slot];
        const float4 thr = P.throughput[slot];
        const uint32_t flags = thr.w < 0.0f ? kUnweightedLight : 0u;
        const FrameConst& f = kBatch ? B.frames[scene] : *fcp;
        const F3 R = miss_path<kAnalytic>(SS, f, W.origin, W.direction, flags, thr.w, V(thr), V(rad));
        P.radiance[slot] = F4(R, 1.0f);
      }
    }
    const unsigned em = __ballot_sync(kFullWarp, emit);
    if (em) {
      if (emit) stage[staged_count + (uint32_t)__popc(em & ((1u << lane) - 1u))] = slot;
      staged_count += (uint32_t)__popc(em);
      if (staged_count >= 32) {
        __syncwarp();
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(hits, 32u);
        base = __shfl_sync(kFullWarp, base, 0);
        Q.hit[base + lane] = stage[lane];
        const uint32_t carry = stage[32 + lane];
        __syncwarp();
        stage[lane] = carry;
        __syncwarp();
        staged_count -= 32;
      }
    }
  }
  __syncwarp();
  if (staged_count) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(hits, staged_count);
    base = __shfl_sync(kFullWarp, base, 0);
    if (lane < staged_count) Q.hit[base + lane] = stage[lane];
  }
  if (kCount) {
    warp_add64(&visits->rays[1], rays);
    warp_add64(&visits->nodes[1], vc.nodes);
    warp_add64(&visits->triangles[1], vc.triangles);
    warp_add64(&visits->instances[1], vc.instances);
  }
}

// Resolve (path_trace.slang:353-385): adds each ended path's sample to its
// pixel and writes the mean; pixels outside the data window keep the clear
// colour.
template <bool kBatch>
__global__ void __launch_bounds__(kBlock) k_wf_resolve(SceneView S,
    const FrameConst* __restrict__ fcp, PathState P, double4* __restrict__ accum,
    float4* __restrict__ color, SceneTable B) {
  const uint32_t index = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t px, py, slot, scene = 0;
  if (kBatch) {
    if (index >= B.total_slots) return;
    slot = index;
    scene = table_scene(B, slot);
    const FrameConst& fb = B.frames[scene];
    const uint32_t local = slot - B.slot_base[scene];
    px = local % fb.width;
    py = local / fb.width;
    if (!frame_rect_contains(fb, px, py)) return;
  } else {
    const uint32_t rect[4] = {fcp->rect[0], fcp->rect[1], fcp->rect[2], fcp->rect[3]};
    if (!tile_pixel(index, rect, px, py)) return;
    slot = py * fcp->width + px;
  }
  const FrameConst& f = kBatch ? B.frames[scene] : *fcp;
  double4 sum = f.accumulated != 0 ? accum[slot] : make_double4(0.0, 0.0, 0.0, 0.0);
  if (f.add_sample) {
    // The wave's samples in order, as one at a time would add them.
    const uint32_t wave = kBatch ? 1u : max(f.wave, 1u);
    for (uint32_t k = 0; k < wave; ++k) sum = add4(sum, P.radiance[k * f.wave_stride + slot]);
    accum[slot] = sum;
  }
  color[slot] = resolve_pixel(kBatch ? B.views[scene] : S, f, px, py, sum);
}

// Ends a sample: totals the queues' rays and advances the sample index.
// The tail (the reference's round scheduler ends its rounds with a tail
// megakernel, vulkan_backend.cpp:3745-3845): the paths still queued for
// bounce `first`, each followed to its end by one thread with the same
// extension trace, scattering and shadow ray, in the same order, as the
// wavefront's rounds, so every path ends with the radiance the rounds would
// give it; the per-bounce queue counts are kept as the rounds keep them.
// Threads take paths from `cursor` one at a time. Long paths then cost one
// launch instead of three per bounce.
template <bool kBatch, bool kAnalytic, bool kFullShading>
__global__ void __launch_bounds__(kBlock, path_loop_blocks(kAnalytic, kFullShading)) k_wf_tail(SceneView S, const FrameConst* __restrict__ fcp, PathState P,
    Queues Q, uint32_t first, uint32_t* __restrict__ cursor, SceneTable B) {
  const uint32_t n = Q.counts[3 * first];
  for (;;) {
    const uint32_t index = atomicAdd(cursor, 1u);
    if (index >= n) return;
    const uint32_t slot = Q.ray[first & 1][index];
    const uint32_t scene = kBatch ? table_scene(B, slot) : 0u;
    const FrameConst& f = kBatch ? B.frames[scene] : *fcp;
    const SceneView& SS = kBatch ? B.views[scene] : S;
    const float4 o = P.origin[slot];
    const float4 d = P.direction[slot];
    const float4 thr = P.throughput[slot];
    const float4 rad = P.radiance[slot];
    F3 ro = V(o), rd = V(d);
    float tmin = o.w, tmax = d.w;
    F3 T = V(thr), R = V(rad);
    float last_pdf = thr.w;
    uint32_t flags = last_pdf < 0.0f ? kUnweightedLight : 0u;
    uint32_t rng = __float_as_uint(rad.w);
    // A path's bounces are bounded by max_bounces (scatter ends it there).
    for (uint32_t bounce = first; bounce <= f.max_bounces; ++bounce) {
      Hit hit;
      if (!trace_closest<false, kFullShading>(SS, ro, rd, tmin, tmax, rng, hit)) {
        R = miss_path<kAnalytic>(SS, f, ro, rd, flags, last_pdf, T, R);
        break;
      }
      atomicAdd(&Q.counts[3 * bounce + 1], 1u);
      F3 no, nd;
      ShadowRequest req;
      const bool cont = scatter<kAnalytic, kFullShading>(SS, f, hit.instance, hit.tri, hit.b1, hit.b2, ro, rd, bounce, T, R,
          last_pdf, flags, rng, no, nd, req, slot);
      if (req.pending) {
        atomicAdd(&Q.counts[3 * bounce + 2], 1u);
        const float tr = trace_shadow<false, kFullShading>(SS, req.origin, req.direction, 0.0f, req.tmax);
        if (tr > 0.0f) R = R + req.throughput * shadow_contribution(req.fl, req.weight, req.pdf, tr);
      }
      if (!cont) break;
      atomicAdd(&Q.counts[3 * (bounce + 1)], 1u);
      if (flags & kUnweightedLight) last_pdf = -1.0f;
      ro = no;
      rd = nd;
      tmin = 0.0f;
      tmax = kFloatMax;
    }
    P.radiance[slot] = F4(R, 1.0f);
  }
}

// The key histogram's exclusive prefix within each block of kSortScanBlock
// bins, in place, and each block's total after the bins.
__global__ void __launch_bounds__(kSortScanBlock) k_sort_scan(uint32_t* __restrict__ bins) {
  __shared__ uint32_t warp_total[kSortScanBlock / 32];
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t i = blockIdx.x * kSortScanBlock + threadIdx.x;
  const uint32_t v = bins[i];
  uint32_t x = v;
  for (unsigned off = 1; off < 32; off <<= 1) {
    const uint32_t y = __shfl_up_sync(kFullWarp, x, off);
    if (lane >= off) x += y;
  }
  if (lane == 31) warp_total[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t t = warp_total[lane];
    for (unsigned off = 1; off < 32; off <<= 1) {
      const uint32_t y = __shfl_up_sync(kFullWarp, t, off);
      if (lane >= off) t += y;
    }
    warp_total[lane] = t;
  }
  __syncthreads();
  const uint32_t before = warp == 0 ? 0u : warp_total[warp - 1];
  bins[i] = before + x - v;
  if (threadIdx.x == kSortScanBlock - 1) bins[kSortBins + blockIdx.x] = before + x;
}

// The queue in key order: each block first scans the block totals; a
// warp's entries of one key take consecutive places from one atomic. The
// entries are `rays[i]`, or the indices i themselves where `rays` is null,
// for i below min(*count, cap).
constexpr int kSortScatterBlock = 256;
static_assert(kSortBlocks == kSortScatterBlock, "one scatter thread per histogram block");
__global__ void __launch_bounds__(kSortScatterBlock) k_sort_scatter(const uint32_t* __restrict__ rays,
    const uint32_t* __restrict__ keys, const uint32_t* __restrict__ count, uint32_t cap, uint32_t* __restrict__ bins,
    uint32_t* __restrict__ sorted) {
  __shared__ uint32_t block_base[kSortBlocks];
  __shared__ uint32_t warp_total[kSortScatterBlock / 32];
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t v = bins[kSortBins + threadIdx.x];
  uint32_t x = v;
  for (unsigned off = 1; off < 32; off <<= 1) {
    const uint32_t y = __shfl_up_sync(kFullWarp, x, off);
    if (lane >= off) x += y;
  }
  if (lane == 31) warp_total[warp] = x;
  __syncthreads();
  uint32_t before = 0;
  for (unsigned w = 0; w < warp; ++w) before += warp_total[w];
  block_base[threadIdx.x] = before + x - v;
  __syncthreads();
  const uint32_t n = min(*count, cap);
  for (uint32_t i = blockIdx.x * kSortScatterBlock + threadIdx.x; i < n; i += gridDim.x * kSortScatterBlock) {
    const uint32_t key = keys[i];
    const unsigned peers = __match_any_sync(__activemask(), key);
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if ((int)lane == leader) base = atomicAdd(&bins[key], (uint32_t)__popc(peers)) + block_base[key / kSortScanBlock];
    base = __shfl_sync(peers, base, leader);
    sorted[base + (uint32_t)__popc(peers & ((1u << lane) - 1u))] = rays != nullptr ? rays[i] : i;
  }
}

__global__ void k_wf_finish(FrameConst* fc, const uint32_t* __restrict__ counts,
    uint32_t max_bounces, RayTotals* totals) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (!fc->add_sample) return;
  unsigned long long ext = 0, sh = 0;
  for (uint32_t b = 0; b <= max_bounces; ++b) {
    if (b != 0) ext += counts[3 * b];
    sh += counts[3 * b + 2];
  }
  totals->camera += (unsigned long long)fc->rect[2] * fc->rect[3] * max(fc->wave, 1u);
  totals->extension += ext;
  totals->shadow += sh;
}

__global__ void k_advance(FrameConst* fc) {
  if (threadIdx.x == 0 && blockIdx.x == 0 && fc->add_sample) {
    fc->sample_index += max(fc->wave, 1u);
    fc->accumulated += max(fc->wave, 1u);
  }
}

// A wave's frame constants: `frame`'s advanced by `offset` samples, covering
// `wave` samples whose slots lie `stride` apart.
__global__ void k_wave_frame(const FrameConst* __restrict__ frame, FrameConst* __restrict__ out, uint32_t offset,
    uint32_t wave, uint32_t stride) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  FrameConst f = *frame;
  if (f.add_sample) {
    f.sample_index += offset;
    f.accumulated += offset;
  }
  f.wave = wave;
  f.wave_stride = stride;
  *out = f;
}

__global__ void k_advance_by(FrameConst* fc, uint32_t samples) {
  if (threadIdx.x == 0 && blockIdx.x == 0 && fc->add_sample) {
    fc->sample_index += samples;
    fc->accumulated += samples;
  }
}

// A batch's k_wf_finish and k_advance: every scene's camera rays, then every
// scene's sample index.
__global__ void k_wf_finish_batch(SceneTable B, const uint32_t* __restrict__ counts, uint32_t max_bounces,
    RayTotals* totals) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  unsigned long long ext = 0, sh = 0, cam = 0;
  for (uint32_t b = 0; b <= max_bounces; ++b) {
    if (b != 0) ext += counts[3 * b];
    sh += counts[3 * b + 2];
  }
  for (uint32_t k = 0; k < B.count; ++k)
    if (B.frames[k].add_sample) cam += (unsigned long long)B.frames[k].rect[2] * B.frames[k].rect[3];
  totals->camera += cam;
  totals->extension += ext;
  totals->shadow += sh;
}

__global__ void k_advance_batch(SceneTable B) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < B.count && B.frames[k].add_sample) {
    B.frames[k].sample_index += 1;
    B.frames[k].accumulated += 1;
  }
}

__global__ void k_fill(float4* color, uint32_t n, float4 v) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) color[i] = v;
}

}  // namespace

namespace {

// Records an event pair around one launch when profiling.
struct Timed {
  SampleProfile* p;
  cudaStream_t s;
  int slot = -1;
  Timed(SampleProfile* profile, cudaStream_t stream, int kind) : p(profile), s(stream) {
    if (p && p->events && p->count < p->capacity) {
      slot = p->count++;
      p->kinds[slot] = kind;
      cudaEventRecord(p->events[2 * slot], s);
    }
  }
  ~Timed() {
    if (slot >= 0) cudaEventRecord(p->events[2 * slot + 1], s);
  }
};

}  // namespace

// Calls f(analytic, textured) with each as a compile-time constant
// (std::true_type / std::false_type), so that a launch takes the
// instantiation without the analytic lights' or texture lookups' code when
// the scene has none.
template <class F>
void with_features(bool analytic, bool full_shading, F&& f) {
  if (analytic && full_shading) f(std::true_type{}, std::true_type{});
  else if (analytic) f(std::true_type{}, std::false_type{});
  else if (full_shading) f(std::false_type{}, std::true_type{});
  else f(std::false_type{}, std::false_type{});
}

void launch_reference_pt(const SceneView& S, const FrameConst* fc, const uint32_t rect[4],
    double4* accum, float4* color, RayTotals* totals, cudaStream_t stream,
    SampleProfile* profile) {
  const uint32_t threads = tile_threads(rect);
  if (threads == 0) return;
  const uint32_t grid = (threads + kBlock - 1) / kBlock;
  Timed t(profile, stream, 0);
  // Counting visits takes the instantiation with every feature's code.
  if (profile && profile->visits) {
    k_reference_pt<true, true, true><<<grid, kBlock, 0, stream>>>(S, fc, accum, color, totals, profile->visits);
    return;
  }
  with_features(S.analytic_count != 0, S.full_shading != 0, [&](auto a, auto x) {
    k_reference_pt<false, decltype(a)::value, decltype(x)::value><<<grid, kBlock, 0, stream>>>(S, fc, accum, color,
        totals, nullptr);
  });
}

// Blocks of a persistent tracing kernel: every resident block on every
// SM (or `blocks_per_sm`), no more than the queue could fill.
// Resident blocks per SM of a kernel at kBlock threads, and the SM count,
// looked up once per process and kernel (every device this library drives
// is an sm_100 part with the same SM count).
int blocks_per_sm(const void* kernel, int& sms) {
  static std::mutex mutex;
  static std::vector<std::pair<const void*, int>> known;
  static int sm_count = 0;
  std::lock_guard<std::mutex> lock(mutex);
  if (sm_count == 0) {
    int device = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device);
  }
  sms = sm_count;
  for (const auto& k : known)
    if (k.first == kernel) return k.second;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, 0);
  known.emplace_back(kernel, per_sm);
  return per_sm;
}

// Blocks of a persistent kernel: every resident block on every SM (or
// `blocks_per_sm`), no more than the queue could fill.
uint32_t persistent_grid(const void* kernel, uint32_t capacity, const TraceTuning& tuning) {
  int sms = 0;
  int per_sm = blocks_per_sm(kernel, sms);
  if (tuning.blocks_per_sm) per_sm = std::min<int>(per_sm, (int)tuning.blocks_per_sm);
  const uint32_t grid = (uint32_t)std::max(1, sms) * (uint32_t)std::max(1, per_sm);
  return std::max(1u, std::min(grid, (capacity + kBlock - 1) / kBlock));
}

uint32_t choose_wavefront_rounds(const uint32_t* counts, uint32_t resident, uint32_t max_bounces) {
  constexpr uint32_t kTailQueue = 65536;
  const uint32_t below = std::max(resident, kTailQueue);
  for (uint32_t b = 1; b <= max_bounces; ++b)
    if (counts[3 * b] < below) return b;
  return max_bounces + 1;
}

uint32_t extension_resident_threads() {
  return persistent_grid((const void*)k_wf_extend<false, false, false, false>, 1u << 30, TraceTuning()) * kBlock;
}

uint32_t wavefront_rounds(uint32_t max_bounces, bool count_visits, uint32_t requested, uint32_t cache_bounce) {
  uint32_t rounds = requested ? requested : LOTUS_WAVEFRONT_ROUNDS;
  // The radiance cache's vertex is shaded in the rounds.
  if (cache_bounce) rounds = std::max(rounds, cache_bounce + 1);
  return count_visits || max_bounces < rounds ? max_bounces + 1 : rounds;
}

void launch_wavefront_sample(const SceneView& S, const FrameConst* fc, const uint32_t rect[4],
    uint32_t width, uint32_t height, uint32_t max_bounces, const PathState& P, const Queues& Q,
    double4* accum, float4* color, RayTotals* totals, cudaStream_t stream,
    SampleProfile* profile, const TraceTuning& tuning, const CacheQueues* cache, cudaEvent_t before_resolve,
    uint32_t wave) {
  CacheQueues C{};
  if (cache && cache->enabled && cache->cache) C = *cache;
  else C.enabled = false;
  (void)width;
  (void)height;
  const uint32_t threads = tile_threads(rect);
  if (threads == 0) return;
  const bool count = profile && profile->visits;
  VisitCounters* visits = profile ? profile->visits : nullptr;
  cudaMemsetAsync(Q.counts, 0, sizeof(uint32_t) * kQueueCounterWords * (size_t)(max_bounces + 2), stream);
  if (C.enabled) cudaMemsetAsync(C.counters, 0, 2 * sizeof(uint32_t), stream);
  uint32_t* fetch = Q.counts + 3 * (size_t)(max_bounces + 2);
  const uint32_t refill = tuning.refill_below ? std::min(tuning.refill_below, 32u) : kDefaultRefillBelow;
  const uint32_t grid_pixels = (threads + kBlock - 1) / kBlock;
  const SceneTable none;
  // The scene's features select the instantiations (counting visits takes
  // the one with every feature's code).
  const bool analytic = S.analytic_count != 0, full_shading = S.full_shading != 0;
  const uint32_t grid_extend = persistent_grid(
      count ? (const void*)k_wf_extend<true, false, true, true> : (const void*)k_wf_extend<false, false, false, false>,
      Q.capacity, tuning);
  const uint32_t grid_shadow = persistent_grid(
      count ? (const void*)k_wf_shadow<true, false, true> : (const void*)k_wf_shadow<false, false, false>, Q.capacity,
      tuning);
  // Shading: up to eight waves of resident blocks, grid-striding over
  // longer queues.
  const uint32_t grid_shade = std::min((Q.capacity + kBlock - 1) / kBlock,
      8u * persistent_grid((const void*)k_wf_shade<false, false, false, false>, Q.capacity, TraceTuning()));
  {
    // One camera thread per pixel of each of the wave's samples.
    Timed t(profile, stream, 0);
    const uint32_t grid_camera = (threads * std::max(wave, 1u) + kBlock - 1) / kBlock;
    if (count) k_wf_camera<true, false, true><<<grid_camera, kBlock, 0, stream>>>(S, fc, P, Q, visits, none);
    else if (full_shading) k_wf_camera<false, false, true><<<grid_camera, kBlock, 0, stream>>>(S, fc, P, Q, nullptr, none);
    else k_wf_camera<false, false, false><<<grid_camera, kBlock, 0, stream>>>(S, fc, P, Q, nullptr, none);
  }
  // Bounces 0 .. rounds - 1 as wavefront rounds; the paths queued for bounce
  // `rounds` (if any can be) go to the tail kernel. Counting visits keeps
  // every bounce in rounds, as the counted kernels are the rounds' own.
  const uint32_t rounds = wavefront_rounds(max_bounces, count, tuning.rounds, C.enabled ? C.bounce : 0u);
  const bool keyed = Q.keys != nullptr && Q.sorted != nullptr && Q.bins != nullptr;
  const uint32_t grid_scatter = persistent_grid((const void*)k_sort_scatter, Q.capacity, TraceTuning());
  for (uint32_t b = 0; b < rounds; ++b) {
    // The queue this round's extension reads: bounce b's rays in key order
    // where shade (b - 1) keyed them.
    const uint32_t* rays = Q.ray[b & 1];
    if (b != 0 && keyed) {
      Timed t(profile, stream, 7);
      k_sort_scan<<<kSortBlocks, kSortScanBlock, 0, stream>>>(Q.bins);
      k_sort_scatter<<<grid_scatter, kSortScatterBlock, 0, stream>>>(Q.ray[b & 1], Q.keys, Q.counts + 3 * b, Q.capacity,
          Q.bins, Q.sorted);
      rays = Q.sorted;
    }
    if (b != 0) {
      Timed t(profile, stream, 1);
      if (count)
        k_wf_extend<true, false, true, true><<<grid_extend, kBlock, 0, stream>>>(S, fc, P, Q, rays, b, fetch + 2 * b,
            refill, visits, none);
      else
        with_features(analytic, full_shading, [&](auto a, auto x) {
          k_wf_extend<false, false, decltype(a)::value, decltype(x)::value><<<grid_extend, kBlock, 0, stream>>>(S, fc,
              P, Q, rays, b, fetch + 2 * b, refill, nullptr, none);
        });
    }
    {
      // Shade keys the rays it queues when a round extends them.
      Queues QS = Q;
      if (keyed && b + 1 < rounds) cudaMemsetAsync(Q.bins, 0, sizeof(uint32_t) * kSortBins, stream);
      else QS.keys = nullptr;
      const bool cache_vertex = C.enabled && b == C.bounce;
      if (cache_vertex && C.query_keys != nullptr)
        cudaMemsetAsync(C.query_bins, 0, sizeof(uint32_t) * kSortBins, stream);
      Timed t(profile, stream, 2);
      with_features(analytic, full_shading, [&](auto a, auto x) {
        if (cache_vertex)
          k_wf_shade<true, false, decltype(a)::value, decltype(x)::value><<<grid_shade, kBlock, 0, stream>>>(S, fc, P,
              QS, b, C, none);
        else
          k_wf_shade<false, false, decltype(a)::value, decltype(x)::value><<<grid_shade, kBlock, 0, stream>>>(S, fc, P,
              QS, b, C, none);
      });
    }
    {
      Timed t(profile, stream, 3);
      if (count)
        k_wf_shadow<true, false, true><<<grid_shadow, kBlock, 0, stream>>>(S, P, Q, b, fetch + 2 * b + 1, refill, visits,
            none);
      else
        if (full_shading)
          k_wf_shadow<false, false, true><<<grid_shadow, kBlock, 0, stream>>>(S, P, Q, b, fetch + 2 * b + 1, refill,
              nullptr, none);
        else
          k_wf_shadow<false, false, false><<<grid_shadow, kBlock, 0, stream>>>(S, P, Q, b, fetch + 2 * b + 1, refill,
              nullptr, none);
    }
    // The training paths' radiance up to their cache vertex's shadow ray.
    if (C.enabled && b == C.bounce)
      k_cache_base<<<(C.train_capacity + kBlock - 1) / kBlock, kBlock, 0, stream>>>(C, P);
  }
  if (rounds <= max_bounces) {
    Timed t(profile, stream, 6);
    uint32_t* cursor = fetch + 2 * (max_bounces + 1);
    with_features(analytic, full_shading, [&](auto a, auto x) {
      const auto kernel = k_wf_tail<false, decltype(a)::value, decltype(x)::value>;
      const uint32_t grid_tail = persistent_grid((const void*)kernel, Q.capacity, tuning);
      kernel<<<grid_tail, kBlock, 0, stream>>>(S, fc, P, Q, rounds, cursor, none);
    });
  }
  if (C.enabled) {
    // The paths that ended into the cache receive its answer; then the
    // training paths' targets train it.
    {
      Timed t(profile, stream, 5);
      const uint32_t* order = nullptr;
      if (C.query_keys != nullptr) {
        k_sort_scan<<<kSortBlocks, kSortScanBlock, 0, stream>>>(C.query_bins);
        k_sort_scatter<<<persistent_grid((const void*)k_sort_scatter, C.query_capacity, TraceTuning()),
            kSortScatterBlock, 0, stream>>>(nullptr, C.query_keys, &C.counters[0], C.query_capacity, C.query_bins,
            C.query_order);
        order = C.query_order;
      }
      launch_cache_infer_records(C.cache->net(), C.cache->grid(), C.queries, C.query_slots, C.query_throughput,
          P.radiance, &C.counters[0], C.query_capacity, stream, order);
    }
    Timed t(profile, stream, 8);
    k_cache_targets<<<(C.train_capacity + kBlock - 1) / kBlock, kBlock, 0, stream>>>(C, P);
    for (uint32_t k = 0; k < C.steps; ++k) {
      launch_cache_train_records(C.cache->net(), C.cache->grid(), C.train, C.train_targets, &C.counters[1],
          C.train_capacity, stream);
      C.cache->adam_step_device(&C.counters[1], C.train_capacity, stream);
    }
  }
  {
    // The accumulation adds samples in order: a sample in flight beside the
    // one before it resolves after that one (and its ray totals).
    if (before_resolve) cudaStreamWaitEvent(stream, before_resolve, 0);
    Timed t(profile, stream, 4);
    k_wf_resolve<false><<<grid_pixels, kBlock, 0, stream>>>(S, fc, P, accum, color, none);
  }
  k_wf_finish<<<1, 32, 0, stream>>>(const_cast<FrameConst*>(fc), Q.counts, max_bounces, totals);
}

__global__ void k_next_frame(const FrameConst* __restrict__ fc, FrameConst* __restrict__ next) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  FrameConst f = *fc;
  if (f.add_sample) {
    f.sample_index += max(f.wave, 1u);
    f.accumulated += max(f.wave, 1u);
  }
  *next = f;
}

void launch_next_frame(const FrameConst* fc, FrameConst* next, cudaStream_t stream) {
  k_next_frame<<<1, 32, 0, stream>>>(fc, next);
}

void launch_wave_frame(const FrameConst* frame, FrameConst* out, uint32_t offset, uint32_t wave, uint32_t stride,
    cudaStream_t stream) {
  k_wave_frame<<<1, 32, 0, stream>>>(frame, out, offset, wave, stride);
}

void launch_advance_by(FrameConst* fc, uint32_t samples, cudaStream_t stream) {
  k_advance_by<<<1, 32, 0, stream>>>(fc, samples);
}

__global__ void k_next_frames(const FrameConst* __restrict__ frames, FrameConst* __restrict__ next, uint32_t count) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  FrameConst f = frames[k];
  if (f.add_sample) {
    f.sample_index += 1;
    f.accumulated += 1;
  }
  next[k] = f;
}

void launch_next_frames(const FrameConst* frames, FrameConst* next, uint32_t count, cudaStream_t stream) {
  k_next_frames<<<(count + 31) / 32, 32, 0, stream>>>(frames, next, count);
}

void launch_advance_batch(const SceneTable& B, cudaStream_t stream) {
  k_advance_batch<<<(B.count + 31) / 32, 32, 0, stream>>>(B);
}

void launch_wavefront_batch(const SceneTable& B, uint32_t max_bounces, const PathState& P, const Queues& Q,
    double4* accum, float4* color, RayTotals* totals, cudaStream_t stream, const TraceTuning& tuning,
    cudaEvent_t before_resolve) {
  if (B.count == 0 || B.total_slots == 0) return;
  const SceneView none_view{};
  const FrameConst* no_frame = nullptr;
  const CacheQueues no_cache;
  cudaMemsetAsync(Q.counts, 0, sizeof(uint32_t) * kQueueCounterWords * (size_t)(max_bounces + 2), stream);
  uint32_t* fetch = Q.counts + 3 * (size_t)(max_bounces + 2);
  const uint32_t refill = tuning.refill_below ? std::min(tuning.refill_below, 32u) : kDefaultRefillBelow;
  const uint32_t grid_slots = (B.total_slots + kBlock - 1) / kBlock;
  const uint32_t grid_extend = persistent_grid((const void*)k_wf_extend<false, true, false, false>, Q.capacity, tuning);
  const uint32_t grid_shadow = persistent_grid((const void*)k_wf_shadow<false, true, true>, Q.capacity, tuning);
  const uint32_t grid_shade = std::min((Q.capacity + kBlock - 1) / kBlock,
      8u * persistent_grid((const void*)k_wf_shade<false, true, false, false>, Q.capacity, TraceTuning()));
  if (B.full_shading) k_wf_camera<false, true, true><<<grid_slots, kBlock, 0, stream>>>(none_view, no_frame, P, Q, nullptr, B);
  else k_wf_camera<false, true, false><<<grid_slots, kBlock, 0, stream>>>(none_view, no_frame, P, Q, nullptr, B);
  const uint32_t rounds = wavefront_rounds(max_bounces, false, tuning.rounds);
  const bool keyed = Q.keys != nullptr && Q.sorted != nullptr && Q.bins != nullptr;
  const uint32_t grid_scatter = persistent_grid((const void*)k_sort_scatter, Q.capacity, TraceTuning());
  for (uint32_t b = 0; b < rounds; ++b) {
    const uint32_t* rays = Q.ray[b & 1];
    if (b != 0 && keyed) {
      k_sort_scan<<<kSortBlocks, kSortScanBlock, 0, stream>>>(Q.bins);
      k_sort_scatter<<<grid_scatter, kSortScatterBlock, 0, stream>>>(Q.ray[b & 1], Q.keys, Q.counts + 3 * b, Q.capacity,
          Q.bins, Q.sorted);
      rays = Q.sorted;
    }
    if (b != 0)
      with_features(B.analytic, B.full_shading, [&](auto a, auto x) {
        k_wf_extend<false, true, decltype(a)::value, decltype(x)::value><<<grid_extend, kBlock, 0, stream>>>(none_view,
            no_frame, P, Q, rays, b, fetch + 2 * b, refill, nullptr, B);
      });
    Queues QS = Q;
    if (keyed && b + 1 < rounds) cudaMemsetAsync(Q.bins, 0, sizeof(uint32_t) * kSortBins, stream);
    else QS.keys = nullptr;
    with_features(B.analytic, B.full_shading, [&](auto a, auto x) {
      k_wf_shade<false, true, decltype(a)::value, decltype(x)::value><<<grid_shade, kBlock, 0, stream>>>(none_view,
          B.frames, P, QS, b, no_cache, B);
    });
    if (B.full_shading)
      k_wf_shadow<false, true, true><<<grid_shadow, kBlock, 0, stream>>>(none_view, P, Q, b, fetch + 2 * b + 1,
          refill, nullptr, B);
    else
      k_wf_shadow<false, true, false><<<grid_shadow, kBlock, 0, stream>>>(none_view, P, Q, b, fetch + 2 * b + 1,
          refill, nullptr, B);
  }
  if (rounds <= max_bounces) {
    uint32_t* cursor = fetch + 2 * (max_bounces + 1);
    with_features(B.analytic, B.full_shading, [&](auto a, auto x) {
      const auto kernel = k_wf_tail<true, decltype(a)::value, decltype(x)::value>;
      const uint32_t grid_tail = persistent_grid((const void*)kernel, Q.capacity, tuning);
      kernel<<<grid_tail, kBlock, 0, stream>>>(none_view, no_frame, P, Q, rounds, cursor, B);
    });
  }
  if (before_resolve) cudaStreamWaitEvent(stream, before_resolve, 0);
  k_wf_resolve<true><<<grid_slots, kBlock, 0, stream>>>(none_view, no_frame, P, accum, color, B);
  k_wf_finish_batch<<<1, 32, 0, stream>>>(B, Q.counts, max_bounces, totals);
  k_advance_batch<<<(B.count + 31) / 32, 32, 0, stream>>>(B);
}

void launch_visibility(const SceneView& S, const VisibilityQueue& queue, uint32_t pass, unsigned char* records,
    uint32_t stride, bool positive, cudaStream_t stream, const TraceTuning& tuning) {
  const uint32_t refill = tuning.refill_below ? std::min(tuning.refill_below, 32u) : kDefaultRefillBelow;
  const uint32_t grid = persistent_grid((const void*)k_visibility, queue.capacity, tuning);
  k_visibility<<<grid, kBlock, 0, stream>>>(S, queue, pass, records, stride, positive ? 1u : 0u, refill);
}

void launch_diagnostic(const SceneView& S, const FrameConst* fc, const uint32_t rect[4], uint32_t output,
    float4* color, cudaStream_t stream) {
  const uint32_t n = rect[2] * rect[3];
  if (n) k_diagnostic<<<(n + kBlock - 1) / kBlock, kBlock, 0, stream>>>(S, fc, output, color);
}

void launch_depth(const SceneView& S, const FrameConst* fc, const uint32_t rect[4], float* depth, uint32_t pixels,
    bool clear, float clear_depth, cudaStream_t stream) {
  if (clear && pixels) k_fill_float<<<(pixels + 255) / 256, 256, 0, stream>>>(depth, pixels, clear_depth);
  const uint32_t n = rect[2] * rect[3];
  if (n) k_depth<<<(n + kBlock - 1) / kBlock, kBlock, 0, stream>>>(S, fc, depth);
}

void launch_advance(FrameConst* fc, cudaStream_t stream) { k_advance<<<1, 32, 0, stream>>>(fc); }

void launch_clear_color(float4* color, uint32_t pixels, float4 value, cudaStream_t stream) {
  if (pixels) k_fill<<<(pixels + 255) / 256, 256, 0, stream>>>(color, pixels, value);
}

}  // namespace lotus
