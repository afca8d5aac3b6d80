// SPDX-License-Identifier: Apache-2.0
// The temporal passes: the primary-surface metadata and its reprojection
// (backend/vulkan/shaders/common/temporal.slang:497-627 in hydra-lotus) and
// ReSTIR DI's initial, temporal and spatial reservoir passes
// (common/restir.slang:163-491); SVGF's are in svgf.cu. One thread per
// pixel; every pass is a separate launch, so each reads only what the
// preceding one finished writing, as the reference's barriers order it.
#include <cooperative_groups.h>
#include <cuda_fp16.h>

#include "../../include/lotus_cuda.h"
#include "temporal_passes.cuh"

namespace lotus {
namespace {

constexpr int kBlock = 128;

__device__ __forceinline__ bool in_rect(const FrameConst& f, uint32_t px, uint32_t py) {
  return px >= f.rect[0] && py >= f.rect[1] && px < f.rect[0] + f.rect[2] && py < f.rect[1] + f.rect[3];
}

// The ReSTIR passes are latency-bound (light and triangle loads, shadow
// rays): six resident blocks per SM hide more of it than registers save.
constexpr int kRestirBlocksPerSm = 6;

// ---------------------------------------------------------------------------
// WriteTemporalSurface (temporal.slang:557-627): the pixel centre's primary
// hit, with a fixed coverage sequence (sample 0).
template <bool kFullShading>
__global__ void __launch_bounds__(kBlock) k_temporal_surface(SceneView S,
    const FrameConst* __restrict__ fcp, const TemporalConst* __restrict__ tcp,
    const TemporalInstance* __restrict__ identities, TemporalPixel* __restrict__ out) {
  const FrameConst& f = *fcp;
  const TemporalConst& tc = *tcp;
  uint32_t px, py;
  if (!pixel_of(blockIdx.x * blockDim.x + threadIdx.x, f.width, f.height, px, py)) return;
  const uint32_t index = py * f.width + px;
  TemporalPixel o = {};
  if (in_rect(f, px, py)) {
    uint32_t rng = seed_random(index, 0);
    const float cx = float(px) + 0.5f, cy = float(py) + 0.5f;
    F3 ro, rd;
    float tmax;
    camera_ray(f, cx * f.ndc[0] + f.ndc[2], cy * f.ndc[1] + f.ndc[3], ro, rd, tmax);
    Hit hit;
    if (trace_closest<false, kFullShading>(S, ro, rd, 0.0f, tmax, rng, hit)) {
      const InstanceShading rec = S.inst_shade[hit.instance];
      const TemporalInstance id = identities[hit.instance];
      const float4* tv = S.tris + kTriStride * (size_t)hit.tri;
      const F3 p0 = V(tv[0]), p1 = V(tv[1]), p2 = V(tv[2]);
      const F3 point = p0 + hit.b1 * (p1 - p0) + hit.b2 * (p2 - p0);
      const F3 world = row_point(rec.m, point);
      const float4 view = mul4(tc.current_view, world.x, world.y, world.z, 1.0f);
      const F3 a = row_point(rec.m, p0), b = row_point(rec.m, p1), c = row_point(rec.m, p2);
      F3 normal = normalize(cross(b - a, c - a));
      if (dot(normal, rd) > 0.0f) normal = -normal;
      const float depth = -view.z / view.w;
      if (finite4(view) && is_finite(normal) && view.w > 0.0f && depth > 0.0f) {
        o.normal_depth = F4(normal, depth);
        o.instance_id = id.instance_id;
        o.material_id = id.material_id;
        o.flags = 1u | id.flags;
        const SurfaceHit sh = reconstruct_hit<kFullShading>(S, hit.instance, hit.tri, hit.b1, hit.b2, rd);
        // The surface summary's albedo (scene.slang:1254-1257).
        const F3 albedo = sh.bsdf.transmission > 0.0f
            ? sh.base_color + sh.bsdf.transmission * (sh.bsdf.transmission_color - sh.base_color)
            : sh.base_color;
        o.albedo = pack_albedo(albedo);
        o.shading_normal = pack_normal(sh.shading_normal);
        if (id.flags & 2u) {
          const F3 pw = row_point(id.previous, point);
          const float4 pv = mul4(tc.previous_view, pw.x, pw.y, pw.z, 1.0f);
          const float4 clip = mul4(tc.previous_world_to_clip, pw.x, pw.y, pw.z, 1.0f);
          const float qx = clip.x / clip.w, qy = clip.y / clip.w, qz = clip.z / clip.w;
          const float pd = -pv.z / pv.w;
          const float ppx = tc.previous_display[0] + (qx * 0.5f + 0.5f) * tc.previous_display[2];
          const float ppy = tc.previous_display[1] + (qy * 0.5f + 0.5f) * tc.previous_display[3];
          const float bx = float(tc.previous_data[0]), by = float(tc.previous_data[1]);
          const float ex = bx + float(tc.previous_data[2]), ey = by + float(tc.previous_data[3]);
          if (finite4(pv) && finite4(clip) && isfinite(ppx) && isfinite(ppy) && isfinite(pd) &&
              pv.w > 0.0f && clip.w > 0.0f && pd > 0.0f && qz >= 0.0f && qz <= 1.0f &&
              qx >= -1.0f && qy >= -1.0f && qx < 1.0f && qy < 1.0f && ppx >= bx && ppy >= by &&
              ppx < ex && ppy < ey)
            o.motion_depth = make_float4(ppx - cx, ppy - cy, pd, 1.0f);
        }
      }
    }
  }
  out[index] = o;
}

// ValidateHistory (temporal.slang:497-522).
__device__ __forceinline__ uint32_t validate_history(const TemporalConst& tc, const TemporalPixel& cur,
    const TemporalPixel& prev) {
  if ((prev.flags & 1u) == 0) return 1u;
  const float* th = tc.validation;
  const F3 n = V(cur.normal_depth), on = V(prev.normal_depth);
  if (!finite4(cur.normal_depth) || !finite4(prev.normal_depth) || !finite4(cur.motion_depth) ||
      !isfinite(th[0]) || !isfinite(th[1]) || !isfinite(th[2]) || !isfinite(th[3]) ||
      cur.normal_depth.w <= 0.0f || prev.normal_depth.w <= 0.0f || cur.motion_depth.z <= 0.0f ||
      th[0] < 0.0f || th[1] < 0.0f || th[2] < -1.0f || th[2] > 1.0f || th[3] < 0.0f ||
      (n.x == 0.0f && n.y == 0.0f && n.z == 0.0f) || (on.x == 0.0f && on.y == 0.0f && on.z == 0.0f))
    return 2u;
  if (cur.instance_id != prev.instance_id) return 3u;
  if (cur.material_id != prev.material_id) return 4u;
  const float mx = cur.motion_depth.x, my = cur.motion_depth.y;
  if (sqrtf(mx * mx + my * my) > th[3]) return 5u;
  if (fabsf(prev.normal_depth.w - cur.motion_depth.z) > th[0] + th[1] * cur.motion_depth.z) return 6u;
  if (dot(normalize(n), normalize(on)) < th[2]) return 7u;
  return 0u;
}

// ReprojectHistory (temporal.slang:524-554): the nearest backward fetch.
__global__ void __launch_bounds__(kBlock) k_reproject(const TemporalConst* __restrict__ tcp,
    const TemporalPixel* __restrict__ current, const TemporalPixel* __restrict__ previous,
    ValidityPixel* __restrict__ out) {
  const TemporalConst& tc = *tcp;
  uint32_t px, py;
  if (!pixel_of(blockIdx.x * blockDim.x + threadIdx.x, tc.width, tc.height, px, py)) return;
  const uint32_t index = py * tc.width + px;
  const TemporalPixel cur = current[index];
  ValidityPixel o = {0u, 0u, 0xffffffffu, 0u};
  if ((cur.flags & 1u) == 0) o.rejection = 1u;
  else if (tc.history == 0) o.rejection = 8u;
  else if ((cur.flags & 2u) == 0) o.rejection = 9u;
  else if ((cur.flags & 4u) == 0) o.rejection = 4u;
  else if (cur.motion_depth.w != 1.0f) o.rejection = 10u;
  else {
    const float ox = float(px) + 0.5f + cur.motion_depth.x;
    const float oy = float(py) + 0.5f + cur.motion_depth.y;
    if (!isfinite(ox) || !isfinite(oy)) o.rejection = 2u;
    else if (ox < 0.0f || oy < 0.0f || ox >= float(tc.width) || oy >= float(tc.height)) o.rejection = 10u;
    else {
      o.previous_index = (uint32_t)oy * tc.width + (uint32_t)ox;
      o.rejection = validate_history(tc, cur, previous[o.previous_index]);
    }
  }
  o.valid = o.rejection == 0u ? 1u : 0u;
  out[index] = o;
}

// ---------------------------------------------------------------------------
// ReSTIR DI.

// A stored surface's closure, by its model.
struct StoredClosure {
  bool gltf;
  Closure preview;
  GltfClosure composed;
};

// ReflectionEvaluate (restir.slang:66-72): ReSTIR's targets are the
// reflection side's.
template <bool kFullShading>
__device__ __forceinline__ F3 reflection_evaluate_side(const StoredClosure& c, F3 wo, F3 wi) {
  if (!(wi.z > 0.0f)) return V(0.0f);
  if (kFullShading && c.gltf) return gltf_evaluate(c.composed, wo, wi);
  return bsdf_evaluate(c.preview, wo, wi);
}

// CandidateContribution (restir.slang:155-161).
template <bool kFullShading>
__device__ __forceinline__ F3 candidate_contribution(const SurfaceHit& sh, const Frame& basis, F3 wo,
    const LightSample& ls, float selection) {
  if (!(ls.pdf > 0.0f) || dot(ls.direction, sh.normal) <= 0.0f) return V(0.0f);
  const F3 wi = basis.to_local(ls.direction);
  const F3 f = wi.z > 0.0f ? surface_evaluate<kFullShading>(sh, wo, wi) : V(0.0f);
  return f * ls.radiance * (selection / ls.pdf);
}

// StoreClosure (restir.slang:78-103): the preview closure's fields, or
// glTF PBR's 22 terms (PackGltfPbrTerms, gltf_pbr.slang:162-188) in the
// same lanes and `extension`. `outgoing.xyz` is already set.
template <bool kFullShading>
__device__ __forceinline__ void store_closure(const SurfaceHit& sh, RestirSurface& s) {
  s.model = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  s.extension = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (kFullShading && sh.gltf) {
    const GltfTerms& g = sh.gltf_terms;
    s.model = make_float4(1.0f, g.e1, g.share, g.f90);
    s.base_alpha = F4(g.base_color, g.alpha);
    s.dielectric_metallic = F4(g.f0, g.metallic);
    s.normal.w = g.transmission;
    s.shading_normal.w = g.coat_scale;
    s.outgoing.w = g.coat_dim;
    s.fresnel = make_float4(g.coat_alpha, g.coat_normal.x, g.coat_normal.y, g.sheen_roughness);
    s.extension = F4(g.sheen_color, g.sheen_dim);
    return;
  }
  const Closure& b = sh.bsdf;
  s.normal.w = b.dielectric_f90;
  s.shading_normal.w = b.thin_walled ? -b.transmission : b.transmission;
  s.outgoing.w = b.smooth ? -b.eta : b.eta;
  s.base_alpha = F4(b.base_color, b.alpha);
  s.dielectric_metallic = F4(b.dielectric_f0, b.metallic);
  s.fresnel = F4(b.f0, b.f90);
}

// LoadClosure (restir.slang:106-150): the glTF closure is rebuilt from its
// terms for the stored outgoing direction (UnpackGltfPbrTerms,
// gltf_pbr.slang:190-214: the coat's normal from its tangent components).
template <bool kFullShading>
__device__ __forceinline__ StoredClosure load_closure(const RestirSurface& s) {
  StoredClosure c;
  c.gltf = kFullShading && (uint32_t)s.model.x == 1u;
  if (kFullShading && c.gltf) {
    GltfTerms g;
    g.base_color = V(s.base_alpha);
    g.alpha = s.base_alpha.w;
    g.metallic = s.dielectric_metallic.w;
    g.e1 = s.model.y;
    g.share = s.model.z;
    g.f0 = V(s.dielectric_metallic);
    g.f90 = s.model.w;
    g.transmission = s.normal.w;
    g.coat_scale = s.shading_normal.w;
    g.coat_dim = s.outgoing.w;
    g.coat_alpha = s.fresnel.x;
    const float tx = s.fresnel.y, ty = s.fresnel.z;
    g.coat_normal = V(tx, ty, sqrtf(fmaxf(1.0f - (tx * tx + ty * ty), 0.0f)));
    g.sheen_color = V(s.extension);
    g.sheen_roughness = s.fresnel.w;
    g.sheen_dim = s.extension.w;
    c.composed = make_gltf_closure(g, V(s.outgoing));
    return c;
  }
  Closure& b = c.preview;
  b.base_color = V(s.base_alpha);
  b.alpha = s.base_alpha.w;
  b.metallic = s.dielectric_metallic.w;
  b.dielectric_f0 = V(s.dielectric_metallic);
  b.dielectric_f90 = s.normal.w;
  b.f0 = V(s.fresnel);
  b.f90 = s.fresnel.w;
  b.transmission = fabsf(s.shading_normal.w);
  b.transmission_color = V(1.0f);
  b.eta = fabsf(s.outgoing.w);
  b.thin_walled = s.shading_normal.w < 0.0f;
  b.smooth = s.outgoing.w < 0.0f;
  return c;
}

// HistoryContribution (restir.slang:256-268).
template <bool kFullShading>
__device__ __forceinline__ F3 history_contribution(const SceneView& S, const RestirSurface& src,
    uint32_t light, const LightSample& ls) {
  if (!(ls.pdf > 0.0f) || dot(ls.direction, V(src.normal)) <= 0.0f) return V(0.0f);
  const StoredClosure b = load_closure<kFullShading>(src);
  const Frame basis = make_frame(V(src.shading_normal));
  return reflection_evaluate_side<kFullShading>(b, V(src.outgoing), basis.to_local(ls.direction)) * ls.radiance *
      (S.lights[light].pdf / ls.pdf);
}

template <bool kFullShading>
__device__ __forceinline__ F3 history_contribution_uv(const SceneView& S, const RestirSurface& src,
    uint32_t light, const float* uv) {
  return history_contribution<kFullShading>(S, src, light,
      reconstruct_reservoir_light<true, kFullShading>(S, light, uv[0], uv[1], V(src.origin)));
}

__device__ __forceinline__ bool same_sample(const RestirPixel& a, const RestirPixel& b) {
  return a.reservoir.sample == b.reservoir.sample && a.uv[0] == b.uv[0] && a.uv[1] == b.uv[1];
}

// HistoryTarget (restir.slang:276-285).
template <bool kFullShading>
__device__ __forceinline__ float history_target(const SceneView& S, const RestirReuse& source,
    const RestirSurface& surface, const RestirPixel& selected, bool& valid) {
  if (same_sample(source.pixel, selected)) {
    valid = isfinite(source.pixel.reservoir.selected_target);
    return source.pixel.reservoir.selected_target;
  }
  const F3 c = history_contribution_uv<kFullShading>(S, surface, selected.reservoir.sample, selected.uv);
  valid = is_finite(c);
  return max_component(c);
}

// Queues pixel `slot`'s shadow ray for pass `pass` of the deferred
// visibility (VisibilityQueue), with its unshadowed contribution and
// normalization; the visibility launch completes the record. One atomic
// per group of lanes that queue together.
__device__ __forceinline__ void queue_visibility(const VisibilityQueue& q, uint32_t pass, uint32_t slot,
    F3 origin, const LightSample& ls, F3 unshadowed, float normalization) {
  namespace cg = cooperative_groups;
  cg::coalesced_group g = cg::coalesced_threads();
  uint32_t base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(&q.counters[2 * pass], g.size());
  base = g.shfl(base, 0);
  const uint32_t i = base + g.thread_rank();
  if (i >= q.capacity) return;  // one ray per pixel at most: never taken
  q.origin[i] = F4(origin, ls.distance);
  q.direction[i] = F4(ls.direction, 0.0f);
  q.slot[i] = slot;
  q.pending[slot] = F4(unshadowed, normalization);
}

// ReceiverVisibility (restir.slang:290-300) and the estimate after it: the
// current sample's visibility when the selected sample is the current one,
// else a queued shadow ray.
__device__ __forceinline__ void receiver_estimate(const VisibilityQueue& q, uint32_t pass, uint32_t slot,
    const RestirPixel& current, F3 origin, const LightSample& ls, F3 unshadowed, float normalization,
    RestirPixel& selected) {
  if (!same_sample(selected, current)) {
    queue_visibility(q, pass, slot, origin, ls, unshadowed, normalization);
    return;
  }
  const float visibility = current.contribution.w;
  const F3 estimate = unshadowed * (visibility * normalization);
  if (!isfinite(normalization) || normalization <= 0.0f || !is_finite(estimate))
    selected.flags |= 2u;
  else
    selected.contribution = F4(estimate, visibility);
}

__device__ __forceinline__ RestirPixel empty_restir_pixel() {
  RestirPixel r;
  r.reservoir = empty_reservoir();
  r.uv[0] = r.uv[1] = 0.0f;
  r.proposal = 0.0f;
  r.flags = 0;
  r.contribution = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  return r;
}

// WriteInitialReservoir (restir.slang:163-233): M candidates streamed over
// the light table at the jittered camera surface, then one shadow ray for
// the selected sample (queued for the deferred visibility, pass 0).
template <bool kFullShading>
__global__ void __launch_bounds__(kBlock, kRestirBlocksPerSm) k_restir_initial(SceneView S,
    const FrameConst* __restrict__ fcp, const TemporalConst* __restrict__ tcp,
    RestirPixel* __restrict__ out, uint4* __restrict__ primary_hit, uint32_t* __restrict__ primary_rng,
    VisibilityQueue VQ) {
  const FrameConst& f = *fcp;
  const TemporalConst& tc = *tcp;
  uint32_t px, py;
  if (!pixel_of(blockIdx.x * blockDim.x + threadIdx.x, f.width, f.height, px, py)) return;
  const uint32_t slot = py * f.width + px;
  RestirPixel r = empty_restir_pixel();
  const bool active = tc.restir_candidates != 0 && in_rect(f, px, py);
  if (active) {
    F3 ro, rd;
    float tmax;
    uint32_t camera_rng;
    start_path(f, px, py, f.sample_index, ro, rd, tmax, camera_rng);
    Hit hit;
    const bool found = trace_closest<false, kFullShading>(S, ro, rd, 0.0f, tmax, camera_rng, hit);
    primary_hit[slot] = found ? make_uint4(hit.instance, hit.tri, __float_as_uint(hit.b1), __float_as_uint(hit.b2))
                              : make_uint4(kNoPrimaryHit, 0u, 0u, 0u);
    primary_rng[slot] = camera_rng;
    if (found) {
      r.flags |= 1u;
      const SurfaceHit sh = reconstruct_hit<kFullShading>(S, hit.instance, hit.tri, hit.b1, hit.b2, rd);
      const Frame basis = make_frame(sh.shading_normal);
      const F3 wo = basis.to_local(-rd);
      const F3 origin = offset_ray_origin(sh.position, sh.normal);
      uint32_t rng = seed_random(slot, f.sample_index ^ 0xD1B54A35u);
      if (tc.max_bounces != 0 && S.light_count != 0) {
        for (uint32_t i = 0; i < tc.restir_candidates; ++i) {
          const float cx = next_random(rng);
          const float cy = next_random(rng);
          const float ux = next_random(rng);
          const float uy = next_random(rng);
          const float random = next_random(rng);
          const uint32_t light = choose_reservoir_light(S, tc.restir_proposal, cx, cy);
          const float proposal = reservoir_proposal_pdf(S, tc.restir_proposal, light);
          const LightSample ls = reconstruct_reservoir_light<true, kFullShading>(S, light, ux, uy, origin);
          const F3 fc = candidate_contribution<kFullShading>(sh, basis, wo, ls, S.lights[light].pdf);
          bool selected;
          if (!isfinite(ls.pdf) || !is_finite(fc) ||
              !stream_candidate(r.reservoir, light, max_component(fc), proposal, random, selected)) {
            r.flags |= 2u;
            break;
          }
          if (selected) {
            r.uv[0] = ux;
            r.uv[1] = uy;
            r.proposal = proposal;
          }
        }
      }
      if ((r.flags & 2u) == 0 && r.reservoir.weight_sum > 0.0f) {
        const LightSample ls = reconstruct_reservoir_light<true, kFullShading>(S, r.reservoir.sample, r.uv[0], r.uv[1], origin);
        queue_visibility(VQ, 0, slot, origin, ls,
            candidate_contribution<kFullShading>(sh, basis, wo, ls, S.lights[r.reservoir.sample].pdf),
            reservoir_normalization(r.reservoir));
      }
    }
  }
  if (r.flags & 2u) atomicMin(&VQ.failed[0], slot);
  out[slot] = r;
}

// WriteTemporalReservoir (restir.slang:302-387).
template <bool kFullShading>
__global__ void __launch_bounds__(kBlock, kRestirBlocksPerSm) k_restir_temporal(SceneView S,
    const FrameConst* __restrict__ fcp, const TemporalConst* __restrict__ tcp,
    const uint4* __restrict__ primary_hit, const TemporalInstance* __restrict__ identities, const RestirPixel* __restrict__ initial,
    const ValidityPixel* __restrict__ validity, const TemporalPixel* __restrict__ surface,
    const RestirReuse* __restrict__ previous, const RestirSurface* __restrict__ previous_surfaces,
    RestirReuse* __restrict__ out, RestirSurface* __restrict__ out_surfaces, VisibilityQueue VQ) {
  const FrameConst& f = *fcp;
  const TemporalConst& tc = *tcp;
  uint32_t px, py;
  if (!pixel_of(blockIdx.x * blockDim.x + threadIdx.x, f.width, f.height, px, py)) return;
  const uint32_t slot = py * f.width + px;
  RestirReuse result = {};
  RestirSurface receiver = {};
  result.pixel = initial[slot];
  result.previous_index = 0xffffffffu;
  result.normalization = reservoir_normalization(result.pixel.reservoir);
  result.supporting_candidates = result.pixel.reservoir.candidate_count;
  const bool active = tc.restir_candidates != 0 && in_rect(f, px, py);
  if (active) {
    F3 ro, rd;
    float tmax;
    uint32_t camera_rng;
    start_path(f, px, py, f.sample_index, ro, rd, tmax, camera_rng);
    // The camera ray's hit as the initial pass traced it.
    const uint4 ph = primary_hit[slot];
    if (ph.x != kNoPrimaryHit) {
      const SurfaceHit sh = reconstruct_hit<kFullShading>(S, ph.x, ph.y, __uint_as_float(ph.z), __uint_as_float(ph.w), rd);
      const Frame basis = make_frame(sh.shading_normal);
      const F3 wo = basis.to_local(-rd);
      const F3 origin = offset_ray_origin(sh.position, sh.normal);
      const float4 view = mul4(tc.current_view, sh.position.x, sh.position.y, sh.position.z, 1.0f);
      receiver.origin = F4(origin, -view.z / view.w);
      receiver.normal = F4(sh.normal, 0.0f);
      receiver.shading_normal = F4(sh.shading_normal, 0.0f);
      receiver.outgoing = F4(wo, 0.0f);
      store_closure<kFullShading>(sh, receiver);
      receiver.instance_id = identities[ph.x].instance_id;
      receiver.material_id = identities[ph.x].material_id;
      const ValidityPixel v = validity[slot];
      const uint32_t previous_index = v.previous_index;
      const bool history = v.valid != 0 && surface[slot].instance_id == receiver.instance_id &&
          surface[slot].material_id == receiver.material_id;
      if (tc.restir_history != 0 && (result.pixel.flags & 2u) == 0 && history) {
        const RestirReuse source = previous[previous_index];
        const RestirSurface& psrc = previous_surfaces[previous_index];
        if ((source.pixel.flags & 1u) != 0 && (source.pixel.flags & 2u) == 0 &&
            psrc.instance_id == receiver.instance_id && psrc.material_id == receiver.material_id) {
          const uint32_t count = min(source.pixel.reservoir.candidate_count, tc.restir_max_history);
          F3 received = V(0.0f);
          if (source.pixel.reservoir.weight_sum > 0.0f) {
            if (source.pixel.reservoir.sample >= S.light_count)
              result.pixel.flags |= 2u;
            else
              received = history_contribution_uv<kFullShading>(S, receiver, source.pixel.reservoir.sample, source.pixel.uv);
          }
          uint32_t rng = seed_random(slot, f.sample_index ^ 0x94D049BBu);
          bool selected;
          if (!is_finite(received) || (result.pixel.flags & 2u) != 0 ||
              !merge_reevaluated(result.pixel.reservoir, source.pixel.reservoir, source.normalization,
                  max_component(received), tc.restir_max_history, next_random(rng), selected)) {
            result.pixel.flags |= 2u;
          } else {
            result.previous_index = previous_index;
            if (selected) {
              result.pixel.uv[0] = source.pixel.uv[0];
              result.pixel.uv[1] = source.pixel.uv[1];
              result.pixel.proposal = source.pixel.proposal;
              result.age = min(source.age, 65535u) + 1u;
            }
            if (result.pixel.reservoir.weight_sum > 0.0f) {
              bool valid_support;
              const float support = history_target<kFullShading>(S, source, psrc, result.pixel, valid_support);
              if (!valid_support) result.pixel.flags |= 2u;
              result.supporting_candidates = initial[slot].reservoir.candidate_count + (support > 0.0f ? count : 0u);
            } else {
              result.supporting_candidates = 0;
            }
            result.normalization = reuse_normalization(result.pixel.reservoir, result.supporting_candidates);
          }
        }
      }
      if ((result.pixel.flags & 2u) == 0 && result.pixel.reservoir.weight_sum > 0.0f) {
        const LightSample ls = reconstruct_reservoir_light<true, kFullShading>(S, result.pixel.reservoir.sample,
            result.pixel.uv[0], result.pixel.uv[1], origin);
        receiver_estimate(VQ, 1, slot, initial[slot], origin, ls,
            history_contribution<kFullShading>(S, receiver, result.pixel.reservoir.sample, ls), result.normalization,
            result.pixel);
      }
    }
  }
  if (result.pixel.flags & 2u) atomicMin(&VQ.failed[1], slot);
  out[slot] = result;
  out_surfaces[slot] = receiver;
}

// SpatialCompatible (restir.slang:392-400).
__device__ __forceinline__ bool spatial_compatible(const RestirSurface& receiver, const RestirReuse& record,
    const RestirSurface& source) {
  return (record.pixel.flags & 3u) == 1u && receiver.origin.w > 0.0f && source.origin.w > 0.0f &&
      receiver.material_id == source.material_id &&
      fabsf(receiver.origin.w - source.origin.w) <= 0.01f + 0.02f * fmaxf(receiver.origin.w, source.origin.w) &&
      dot(V(receiver.normal), V(source.normal)) >= 0.9f &&
      dot(V(receiver.shading_normal), V(source.shading_normal)) >= 0.9f;
}

// The spatial pass's neighbour offsets: the reference's four axis
// neighbours at the radius (restir.slang:408-410), or `count` distinct
// offsets drawn uniformly from the disk of the radius, the centre excluded
// (no counterpart in the reference): each the first of up to kDiskTries
// draws of an offset in the enclosing square that falls inside the disk
// and was not drawn before, from the pixel's own stream for this purpose.
// Returns how many offsets there are.
constexpr int kMaxNeighbours = LOTUS_MAX_SPATIAL_NEIGHBOURS;
constexpr int kDiskTries = 16;

__device__ __forceinline__ int spatial_offsets(uint32_t slot, uint32_t sample_index, int radius, uint32_t count,
    int ox[kMaxNeighbours], int oy[kMaxNeighbours]) {
  if (count == 0) {
    ox[0] = -radius, oy[0] = 0;
    ox[1] = radius, oy[1] = 0;
    ox[2] = 0, oy[2] = -radius;
    ox[3] = 0, oy[3] = radius;
    return 4;
  }
  uint32_t rng = seed_random(slot, sample_index ^ 0x5BD1E995u);
  const float side = float(2 * radius + 1);
  int n = 0;
  for (uint32_t i = 0; i < count; ++i) {
    for (int t = 0; t < kDiskTries; ++t) {
      const int dx = min((int)(next_random(rng) * side), 2 * radius) - radius;
      const int dy = min((int)(next_random(rng) * side), 2 * radius) - radius;
      if ((dx == 0 && dy == 0) || dx * dx + dy * dy > radius * radius) continue;
      bool seen = false;
      for (int k = 0; k < n; ++k) seen = seen || (ox[k] == dx && oy[k] == dy);
      if (seen) continue;
      ox[n] = dx;
      oy[n] = dy;
      ++n;
      break;
    }
  }
  return n;
}

// WriteSpatialReservoir (restir.slang:402-491): the neighbours above,
// merged with support correction.
template <bool kFullShading>
__global__ void __launch_bounds__(kBlock, kRestirBlocksPerSm) k_restir_spatial(SceneView S,
    const FrameConst* __restrict__ fcp, const TemporalConst* __restrict__ tcp,
    const RestirReuse* __restrict__ temporal, const RestirSurface* __restrict__ surfaces,
    RestirReuse* __restrict__ out, uint4* __restrict__ out_sources, VisibilityQueue VQ) {
  const FrameConst& f = *fcp;
  const TemporalConst& tc = *tcp;
  uint32_t px, py;
  if (!pixel_of(blockIdx.x * blockDim.x + threadIdx.x, f.width, f.height, px, py)) return;
  const uint32_t slot = py * f.width + px;
  const RestirReuse centre = temporal[slot];
  const RestirSurface receiver = surfaces[slot];
  RestirReuse result = centre;
  uint32_t sources[kMaxNeighbours];
  for (int i = 0; i < kMaxNeighbours; ++i) sources[i] = 0xffffffffu;
  int ox[kMaxNeighbours], oy[kMaxNeighbours];
  const int neighbours = (centre.pixel.flags & 3u) == 1u
      ? spatial_offsets(slot, f.sample_index, (int)tc.restir_radius, tc.restir_neighbours, ox, oy) : 0;
  if ((centre.pixel.flags & 3u) == 1u) {
    uint32_t accepted = 0;
    for (int i = 0; i < neighbours; ++i) {
      const int nx = (int)px + ox[i], ny = (int)py + oy[i];
      if (nx < 0 || ny < 0 || nx >= (int)f.width || ny >= (int)f.height) continue;
      const uint32_t index = (uint32_t)ny * f.width + (uint32_t)nx;
      if (spatial_compatible(receiver, temporal[index], surfaces[index])) {
        sources[i] = index;
        ++accepted;
      }
    }
    if (accepted != 0) {
      result.pixel.reservoir = empty_reservoir();
      bool selected;
      if (!merge_reevaluated(result.pixel.reservoir, centre.pixel.reservoir, centre.normalization,
              centre.pixel.reservoir.selected_target, 0xffffffffu, 0.0f, selected))
        result.pixel.flags |= 2u;
      uint32_t rng = seed_random(slot, f.sample_index ^ 0x369DEA0Fu);
      for (int i = 0; i < neighbours; ++i) {
        if (sources[i] == 0xffffffffu) continue;
        const RestirReuse source = temporal[sources[i]];
        F3 received = V(0.0f);
        if (source.pixel.reservoir.weight_sum > 0.0f)
          received = history_contribution_uv<kFullShading>(S, receiver, source.pixel.reservoir.sample, source.pixel.uv);
        if (!is_finite(received) ||
            !merge_reevaluated(result.pixel.reservoir, source.pixel.reservoir, source.normalization,
                max_component(received), tc.restir_max_history, next_random(rng), selected)) {
          result.pixel.flags |= 2u;
          break;
        }
        if (selected) {
          result.pixel.uv[0] = source.pixel.uv[0];
          result.pixel.uv[1] = source.pixel.uv[1];
          result.pixel.proposal = source.pixel.proposal;
          result.age = source.age;
        }
      }
      result.supporting_candidates = 0;
      result.pixel.contribution = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      if ((result.pixel.flags & 2u) == 0 && result.pixel.reservoir.weight_sum > 0.0f) {
        result.supporting_candidates = centre.pixel.reservoir.candidate_count;
        for (int i = 0; i < neighbours; ++i) {
          if (sources[i] == 0xffffffffu) continue;
          const RestirReuse source = temporal[sources[i]];
          bool valid_support;
          const float support = history_target<kFullShading>(S, source, surfaces[sources[i]], result.pixel, valid_support);
          if (!valid_support) result.pixel.flags |= 2u;
          if (support > 0.0f)
            result.supporting_candidates += min(source.pixel.reservoir.candidate_count, tc.restir_max_history);
        }
      }
      result.normalization = reuse_normalization(result.pixel.reservoir, result.supporting_candidates);
      if ((result.pixel.flags & 2u) == 0 && result.pixel.reservoir.weight_sum > 0.0f) {
        const LightSample ls = reconstruct_reservoir_light<true, kFullShading>(S, result.pixel.reservoir.sample,
            result.pixel.uv[0], result.pixel.uv[1], V(receiver.origin));
        receiver_estimate(VQ, 2, slot, centre.pixel, V(receiver.origin), ls,
            history_contribution<kFullShading>(S, receiver, result.pixel.reservoir.sample, ls), result.normalization,
            result.pixel);
      }
    }
  }
  if (result.pixel.flags & 2u) atomicMin(&VQ.failed[2], slot);
  out[slot] = result;
  out_sources[slot] = make_uint4(sources[0], sources[1], sources[2], sources[3]);
}

inline uint32_t grid(uint32_t n) { return (n + kBlock - 1) / kBlock; }

}  // namespace

void launch_temporal_surface(const SceneView& S, const FrameConst* fc, const TemporalConst* tc,
    const TemporalInstance* ids, TemporalPixel* out, uint32_t pixels, cudaStream_t s) {
  if (S.full_shading) k_temporal_surface<true><<<grid(pixels), kBlock, 0, s>>>(S, fc, tc, ids, out);
  else k_temporal_surface<false><<<grid(pixels), kBlock, 0, s>>>(S, fc, tc, ids, out);
}

void launch_reproject(const TemporalConst* tc, const TemporalPixel* current, const TemporalPixel* previous,
    ValidityPixel* out, uint32_t pixels, cudaStream_t s) {
  k_reproject<<<grid(pixels), kBlock, 0, s>>>(tc, current, previous, out);
}

void launch_restir_initial(const SceneView& S, const FrameConst* fc, const TemporalConst* tc,
    RestirPixel* out, uint4* primary_hit, uint32_t* primary_rng, const VisibilityQueue& vq, uint32_t pixels,
    cudaStream_t s) {
  if (S.full_shading) k_restir_initial<true><<<grid(pixels), kBlock, 0, s>>>(S, fc, tc, out, primary_hit, primary_rng, vq);
  else k_restir_initial<false><<<grid(pixels), kBlock, 0, s>>>(S, fc, tc, out, primary_hit, primary_rng, vq);
}

void launch_restir_temporal(const SceneView& S, const FrameConst* fc, const TemporalConst* tc,
    const uint4* primary_hit, const TemporalInstance* ids, const RestirPixel* initial,
    const ValidityPixel* validity, const TemporalPixel* surface, const RestirReuse* previous,
    const RestirSurface* previous_surfaces, RestirReuse* out, RestirSurface* out_surfaces,
    const VisibilityQueue& vq, uint32_t pixels, cudaStream_t s) {
  if (S.full_shading)
    k_restir_temporal<true><<<grid(pixels), kBlock, 0, s>>>(S, fc, tc, primary_hit, ids, initial, validity, surface,
        previous, previous_surfaces, out, out_surfaces, vq);
  else
    k_restir_temporal<false><<<grid(pixels), kBlock, 0, s>>>(S, fc, tc, primary_hit, ids, initial, validity, surface,
        previous, previous_surfaces, out, out_surfaces, vq);
}

void launch_restir_spatial(const SceneView& S, const FrameConst* fc, const TemporalConst* tc,
    const RestirReuse* temporal, const RestirSurface* surfaces, RestirReuse* out, uint4* sources,
    const VisibilityQueue& vq, uint32_t pixels, cudaStream_t s) {
  if (S.full_shading) k_restir_spatial<true><<<grid(pixels), kBlock, 0, s>>>(S, fc, tc, temporal, surfaces, out, sources, vq);
  else k_restir_spatial<false><<<grid(pixels), kBlock, 0, s>>>(S, fc, tc, temporal, surfaces, out, sources, vq);
}

}  // namespace lotus
