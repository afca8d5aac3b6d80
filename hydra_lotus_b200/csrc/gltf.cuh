// SPDX-License-Identifier: Apache-2.0
// MaterialX's glTF PBR surface on the device (backend/vulkan/shaders/bsdf/
// gltf_pbr.slang, composed.slang and lobes.slang in hydra-lotus):
//
//   layer(clearcoat, layer(sheen, mix(layer(generalized_schlick(f0, f90),
//       mix(lambert(base_color), transmission, transmission)),
//       generalized_schlick(base_color, 1), metallic)))
//
// The reference builds it as a general list of lobes with mix, scale and
// layer operations (a composed closure, up to six lobes). Here the list's
// shape is fixed, so each lobe has a slot in the reference's build order
// (coat, sheen, dielectric reflection, diffuse, thin transmission, metal)
// and its weight is the product of the factors the operations would apply
// to it, in the order they apply them: the values equal the general
// closure's bit for bit (the oracle builds the general list). The
// integrators evaluate, give densities for and sample it in the shading
// frame, as they do UsdPreviewSurface's closure.
#pragma once

#include "albedo.cuh"
#include "bsdf.cuh"

namespace lotus {

constexpr float kGltfClearcoatIndex = 1.5f;
constexpr float kMinSheenRoughness = 0.005f;
// A lobe with a positive estimate is chosen at least this often, before
// renormalization (composed.slang's kSelectionFloor).
constexpr float kSelectionFloor = 0.05f;

// The lobe slots, in the order the reference's builder appends them.
constexpr uint32_t kGltfCoat = 0, kGltfSheen = 1, kGltfSpecular = 2, kGltfDiffuse = 3,
                   kGltfTransmit = 4, kGltfMetal = 5, kGltfLobes = 6;

// GltfPbrInputs (gltf_pbr.slang:33-52): the model's inputs at a hit.
struct GltfInputs {
  F3 base_color;
  float roughness;
  float metallic;
  float dielectric_f0;  // ((1 - ior) / (1 + ior))^2
  float specular;
  F3 specular_color;
  float transmission;
  float clearcoat;
  float clearcoat_roughness;
  F3 clearcoat_normal;  // unit, in the shading frame
  F3 sheen_color;
  float sheen_roughness;
};

// GltfPbrTerms (gltf_pbr.slang:76-104): the inputs reduced to what the
// lobes read, with every table value at the outgoing direction.
struct GltfTerms {
  F3 base_color;
  float alpha;
  float metallic;
  float e1;
  float share;
  F3 f0;
  float f90;
  float transmission;
  float coat_scale;
  float coat_dim;
  float coat_alpha;
  F3 coat_normal;
  F3 sheen_color;
  float sheen_roughness;
  float sheen_dim;
};

// MakeGltfPbrTerms (gltf_pbr.slang:106-157).
__device__ __forceinline__ GltfTerms make_gltf_terms(const GltfInputs& in, F3 wo,
    const float* __restrict__ tables) {
  GltfTerms t;
  t.base_color = in.base_color;
  t.alpha = fmaxf(in.roughness * in.roughness, kMinAlpha);
  t.metallic = in.metallic;
  t.e1 = 0.0f;
  t.share = 0.0f;
  if (wo.z > 0.0f) albedo::ggx_and_share(tables, wo.z, t.alpha, t.e1, t.share);
  const F3 tinted = in.specular_color * in.dielectric_f0;
  t.f0 = V(saturate(tinted.x), saturate(tinted.y), saturate(tinted.z)) * in.specular;
  t.f90 = in.specular;
  t.transmission = in.transmission;
  t.coat_scale = 0.0f;
  t.coat_dim = 0.0f;
  t.coat_alpha = fmaxf(in.clearcoat_roughness * in.clearcoat_roughness, kMinAlpha);
  t.coat_normal = in.clearcoat_normal.z > 0.0f ? in.clearcoat_normal : V(0.0f, 0.0f, 1.0f);
  const float coat_cos = dot(wo, t.coat_normal);
  if (in.clearcoat > 0.0f && coat_cos > 0.0f) {
    const float reflected = albedo::dielectric(tables, coat_cos, t.coat_alpha, kGltfClearcoatIndex, false);
    const float coat_e1 = albedo::ggx(tables, coat_cos, t.coat_alpha);
    const float root = (1.0f - kGltfClearcoatIndex) / (1.0f + kGltfClearcoatIndex);
    float compensation = 1.0f;
    if (coat_e1 > 0.0f) compensation += root * root * (1.0f - coat_e1) / coat_e1;
    t.coat_scale = in.clearcoat * compensation;
    t.coat_dim = saturate(t.coat_scale * reflected);
  }
  t.sheen_color = in.sheen_color;
  t.sheen_roughness = fmaxf(in.sheen_roughness * in.sheen_roughness, kMinSheenRoughness);
  t.sheen_dim = 0.0f;
  const float sheen = max_component(in.sheen_color);
  if (sheen > 0.0f && wo.z > 0.0f) {
    const float e = albedo::sheen(tables, wo.z, t.sheen_roughness);
    if (e > 1.0f) t.sheen_color = in.sheen_color * (1.0f / e);
    t.sheen_dim = saturate(sheen * fminf(e, 1.0f));
  }
  return t;
}

// The built closure: each slot's lobe parameters, weight, compensation and
// selection probability for the outgoing direction it was built for.
struct GltfClosure {
  uint32_t present;  // a bit per slot
  F3 base_color;     // the diffuse lobe's albedo, the metal's f0, the transmission's tint
  float alpha;       // GGX alpha of the three base lobes
  F3 f0;             // the dielectric reflection's Schlick colours
  float f90;
  F3 coat_normal;
  float coat_alpha;
  float sheen_roughness;
  float w_coat;
  F3 w_sheen;
  float w_specular;
  float w_diffuse;
  F3 w_transmit;
  float w_metal;
  F3 c_specular;  // multiple-scattering compensation
  float c_transmit;
  F3 c_metal;
  float p[kGltfLobes];
};

// MakeGltfPbrClosure (gltf_pbr.slang:230-290) over ComposedAdd* and the
// mix and layer operations (composed.slang:131-308), in their order.
__device__ __forceinline__ GltfClosure make_gltf_closure(const GltfTerms& t, F3 wo) {
  GltfClosure c;
  c.present = 0;
  c.base_color = t.base_color;
  c.alpha = fmaxf(t.alpha, kMinAlpha);
  c.f0 = t.f0;
  c.f90 = t.f90;
  c.coat_normal = t.coat_normal;
  c.coat_alpha = fmaxf(t.coat_alpha, kMinAlpha);
  c.sheen_roughness = fmaxf(t.sheen_roughness, kMinSheenRoughness);
  c.w_coat = 0.0f;
  c.w_sheen = V(0.0f);
  c.w_specular = 0.0f;
  c.w_diffuse = 0.0f;
  c.w_transmit = V(0.0f);
  c.w_metal = 0.0f;
  c.c_specular = V(1.0f);
  c.c_transmit = 1.0f;
  c.c_metal = V(1.0f);
  // Each lobe's albedo toward wo as a layer above it sees it, and its
  // estimate (the basis of its selection probability).
  float coat_albedo = 0.0f, sheen_albedo = 0.0f, transmit_estimate = 0.0f;
  F3 specular_albedo = V(0.0f), diffuse_albedo = V(0.0f), metal_albedo = V(0.0f);
  const bool up = wo.z > 0.0f;  // wo above the base lobes' normal
  if (t.coat_scale > 0.0f) {
    c.present |= 1u << kGltfCoat;
    c.w_coat = t.coat_scale;
    coat_albedo = t.coat_dim / t.coat_scale;
  }
  if (t.sheen_dim > 0.0f) {
    c.present |= 1u << kGltfSheen;
    c.w_sheen = t.sheen_color;
    sheen_albedo = t.sheen_dim / max_component(t.sheen_color);
  }
  const bool dielectric = t.metallic < 1.0f;
  if (dielectric && t.f90 > 0.0f) {
    c.present |= 1u << kGltfSpecular;
    c.w_specular = 1.0f;
    if (up) {
      if (t.e1 > 0.0f) c.c_specular = V(1.0f) + c.f0 * ((1.0f - t.e1) / t.e1);
      specular_albedo = (c.f0 * (t.e1 - t.share) + V(c.f90 * t.share)) * c.c_specular;
    }
  }
  if (dielectric && t.transmission < 1.0f) {
    c.present |= 1u << kGltfDiffuse;
    c.w_diffuse = 1.0f;
    diffuse_albedo = up ? c.base_color : V(0.0f);
  }
  if (dielectric && t.transmission > 0.0f) {
    c.present |= 1u << kGltfTransmit;
    if (up) {
      if (t.e1 > 0.0f) c.c_transmit = 1.0f + 1.0f * ((1.0f - t.e1) / t.e1);
      transmit_estimate = (1.0f * (t.e1 - t.share) + 1.0f * t.share) * c.c_transmit;
    }
    c.w_transmit = V(1.0f) * c.base_color;
  }
  if (t.transmission > 0.0f) {
    // mix(diffuse, transmission, transmission)
    c.w_diffuse = c.w_diffuse * (1.0f - t.transmission);
    c.w_transmit = c.w_transmit * t.transmission;
  }
  {
    // The dielectric's reflection over the diffuse and transmitted base,
    // dimming it by its largest channel.
    const F3 top = c.w_specular * specular_albedo;
    const float f = saturate(1.0f - max_component(top));
    c.w_diffuse = c.w_diffuse * f;
    c.w_transmit = c.w_transmit * f;
  }
  if (t.metallic > 0.0f) {
    c.present |= 1u << kGltfMetal;
    c.w_metal = 1.0f;
    if (up) {
      if (t.e1 > 0.0f) c.c_metal = V(1.0f) + c.base_color * ((1.0f - t.e1) / t.e1);
      metal_albedo = (c.base_color * (t.e1 - t.share) + V(1.0f * t.share)) * c.c_metal;
    }
  }
  {
    // mix(dielectric base, metal, metallic)
    const float m = 1.0f - t.metallic;
    c.w_specular = c.w_specular * m;
    c.w_diffuse = c.w_diffuse * m;
    c.w_transmit = c.w_transmit * m;
    c.w_metal = c.w_metal * t.metallic;
  }
  {
    // The sheen over everything below it, by its largest channel.
    const F3 top = c.w_sheen * sheen_albedo;
    const float f = saturate(1.0f - max_component(top));
    c.w_specular = c.w_specular * f;
    c.w_diffuse = c.w_diffuse * f;
    c.w_transmit = c.w_transmit * f;
    c.w_metal = c.w_metal * f;
  }
  {
    // The coat over the sheen and everything below.
    const float f = saturate(1.0f - c.w_coat * coat_albedo);
    c.w_sheen = c.w_sheen * f;
    c.w_specular = c.w_specular * f;
    c.w_diffuse = c.w_diffuse * f;
    c.w_transmit = c.w_transmit * f;
    c.w_metal = c.w_metal * f;
  }
  // ComposedFinalize (composed.slang:329-353): probabilities proportional
  // to the estimates, floored, renormalized.
  float e[kGltfLobes];
  e[kGltfCoat] = c.w_coat * coat_albedo;
  e[kGltfSheen] = max_component(c.w_sheen * sheen_albedo);
  e[kGltfSpecular] = max_component(c.w_specular * specular_albedo);
  e[kGltfDiffuse] = max_component(c.w_diffuse * diffuse_albedo);
  e[kGltfTransmit] = max_component(c.w_transmit * transmit_estimate);
  e[kGltfMetal] = max_component(c.w_metal * metal_albedo);
  float total = 0.0f;
#pragma unroll
  for (uint32_t k = 0; k < kGltfLobes; ++k) {
    c.p[k] = (c.present >> k & 1u) && e[k] > 0.0f ? e[k] : 0.0f;
    total += c.p[k];
  }
  if (!(total > 0.0f)) return c;
  float floored = 0.0f;
#pragma unroll
  for (uint32_t k = 0; k < kGltfLobes; ++k)
    if (c.p[k] > 0.0f) {
      c.p[k] = fmaxf(c.p[k] / total, kSelectionFloor);
      floored += c.p[k];
    }
#pragma unroll
  for (uint32_t k = 0; k < kGltfLobes; ++k) c.p[k] = c.p[k] / floored;
  return c;
}

// --- Lobes (lobes.slang:238-508), each in the frame about its normal --------

// GGX reflection's D * G2 / (4 cos(theta_o)) with the height-correlated
// Smith term.
__device__ __forceinline__ float gltf_ggx_reflection(F3 wo, F3 wi, F3 h, float alpha) {
  const float g2 = 1.0f / (1.0f + ggx_lambda(wo, alpha) + ggx_lambda(wi, alpha));
  return ggx_d(h, alpha) * g2 / (4.0f * wo.z);
}

__device__ __forceinline__ float gltf_ggx_reflection_pdf(F3 wo, F3 h, float alpha) {
  const float g1 = 1.0f / (1.0f + ggx_lambda(wo, alpha));
  return ggx_d(h, alpha) * g1 / (4.0f * wo.z);
}

// A GgxSchlick lobe's f cos(theta_i): colour f0 and f90, compensation c;
// `mirrored` reflects through the tangent plane (thin transmission).
__device__ __forceinline__ F3 gltf_schlick_value(F3 f0, F3 f90, F3 comp, float alpha, bool mirrored,
    F3 wo, F3 wi) {
  const F3 wr = mirrored ? V(wi.x, wi.y, -wi.z) : wi;
  if (!(wr.z > 0.0f)) return V(0.0f);
  const F3 h = normalize(wo + wr);
  const float weight = lpow5(saturate(1.0f - dot(wo, h)));
  const F3 fresnel = f0 * (1.0f - weight) + f90 * weight;
  return fresnel * comp * gltf_ggx_reflection(wo, wr, h, alpha);
}

__device__ __forceinline__ float gltf_schlick_pdf(float alpha, bool mirrored, F3 wo, F3 wi) {
  const F3 wr = mirrored ? V(wi.x, wi.y, -wi.z) : wi;
  return wr.z > 0.0f ? gltf_ggx_reflection_pdf(wo, normalize(wo + wr), alpha) : 0.0f;
}

// The Conty-Kulla sheen, white, uncompensated: D / (4 (cos_i + cos_o -
// cos_i cos_o)) cos_i with D = (2 + 1/r) sin(theta_h)^(1/r) / (2 pi).
__device__ __forceinline__ float gltf_sheen_value(float roughness, F3 wo, F3 wi) {
  if (!(wi.z > 0.0f)) return 0.0f;
  const F3 h = normalize(wo + wi);
  const float inverse = 1.0f / roughness;
  const float sin2 = fmaxf(1.0f - h.z * h.z, 0.0f);
  const float d = (2.0f + inverse) * lpow(sin2, 0.5f * inverse) / (2.0f * kPi);
  return 1.0f * 1.0f * (d * wi.z / (4.0f * (wi.z + wo.z - wi.z * wo.z)));
}

// The coat: a rough dielectric of index 1.5 that reflects only.
__device__ __forceinline__ float gltf_coat_value(float alpha, F3 wo, F3 wi) {
  if (!(wi.z > 0.0f)) return 0.0f;
  const F3 h = normalize(wo + wi);
  return 1.0f * 1.0f * (fresnel_dielectric(dot(wo, h), kGltfClearcoatIndex) *
      gltf_ggx_reflection(wo, wi, h, alpha));
}

__device__ __forceinline__ float gltf_coat_pdf(float alpha, F3 wo, F3 wi) {
  if (!(wi.z > 0.0f)) return 0.0f;
  return 1.0f * gltf_ggx_reflection_pdf(wo, normalize(wo + wi), alpha);
}

// --- The closure (composed.slang:355-445) -------------------------------------

// Whether slot k scatters into wi's hemisphere of the shading frame: the
// thin transmission into the lower one, every other lobe into the upper.
__device__ __forceinline__ bool gltf_scatters_toward(uint32_t k, F3 wi) {
  return k == kGltfTransmit ? wi.z < 0.0f : wi.z > 0.0f;
}

// The coat's f cos(theta_i) in its frame; 0 where wo lies below its normal.
__device__ __forceinline__ float gltf_coat_term(const GltfClosure& c, F3 wo, F3 wi) {
  const Frame f = make_frame(c.coat_normal);
  const F3 lo = f.to_local(wo);
  return lo.z > 0.0f ? gltf_coat_value(c.coat_alpha, lo, f.to_local(wi)) : 0.0f;
}

// f(wo, wi) |cos(theta_i)| summed over the slots in order.
__device__ __forceinline__ F3 gltf_evaluate(const GltfClosure& c, F3 wo, F3 wi) {
  F3 value = V(0.0f);
  if ((c.present & (1u << kGltfCoat)) && wi.z > 0.0f)
    value = value + V(c.w_coat * 1.0f * gltf_coat_term(c, wo, wi));
  // The base's lobes lie about the shading normal.
  if (!(wo.z > 0.0f)) return value;
  if ((c.present & (1u << kGltfSheen)) && wi.z > 0.0f)
    value = value + c.w_sheen * 1.0f * gltf_sheen_value(c.sheen_roughness, wo, wi);
  if ((c.present & (1u << kGltfSpecular)) && wi.z > 0.0f)
    value = value + V(c.w_specular) * 1.0f *
        gltf_schlick_value(c.f0, V(c.f90), c.c_specular, c.alpha, false, wo, wi);
  if ((c.present & (1u << kGltfDiffuse)) && wi.z > 0.0f)
    value = value + V(c.w_diffuse) * 1.0f * (c.base_color * (wi.z / kPi));
  if ((c.present & (1u << kGltfTransmit)) && wi.z < 0.0f)
    value = value + c.w_transmit * 1.0f *
        gltf_schlick_value(V(1.0f), V(1.0f), V(c.c_transmit), c.alpha, true, wo, wi);
  if ((c.present & (1u << kGltfMetal)) && wi.z > 0.0f)
    value = value + V(c.w_metal) * 1.0f *
        gltf_schlick_value(c.base_color, V(1.0f), c.c_metal, c.alpha, false, wo, wi);
  return value;
}

// The density with which gltf_sample returns wi: sum_k p_k pdf_k.
__device__ __forceinline__ float gltf_pdf(const GltfClosure& c, F3 wo, F3 wi) {
  float pdf = 0.0f;
  if (c.p[kGltfCoat] > 0.0f && wi.z > 0.0f) {
    const Frame f = make_frame(c.coat_normal);
    const F3 lo = f.to_local(wo);
    if (lo.z > 0.0f) pdf += c.p[kGltfCoat] * gltf_coat_pdf(c.coat_alpha, lo, f.to_local(wi));
  }
  if (!(wo.z > 0.0f)) return pdf;
  if (c.p[kGltfSheen] > 0.0f && wi.z > 0.0f) pdf += c.p[kGltfSheen] * (1.0f / (2.0f * kPi));
  if (c.p[kGltfSpecular] > 0.0f && wi.z > 0.0f)
    pdf += c.p[kGltfSpecular] * gltf_schlick_pdf(c.alpha, false, wo, wi);
  if (c.p[kGltfDiffuse] > 0.0f && wi.z > 0.0f) pdf += c.p[kGltfDiffuse] * (wi.z / kPi);
  if (c.p[kGltfTransmit] > 0.0f && wi.z < 0.0f)
    pdf += c.p[kGltfTransmit] * gltf_schlick_pdf(c.alpha, true, wo, wi);
  if (c.p[kGltfMetal] > 0.0f && wi.z > 0.0f) pdf += c.p[kGltfMetal] * gltf_schlick_pdf(c.alpha, false, wo, wi);
  return pdf;
}

// ComposedSample (composed.slang:400-445): one lobe chosen with u.z, then
// its direction from u.xy; the weight is the mixture's f cos / pdf.
__device__ __forceinline__ bool gltf_sample(const GltfClosure& c, F3 wo, F3 u, BsdfSample& s) {
  s.wi = V(0.0f, 0.0f, 1.0f);
  s.weight = V(0.0f);
  s.pdf = 0.0f;
  s.delta = false;
  s.transmitted = false;
  uint32_t chosen = kGltfLobes;
  float end = 0.0f;
  // Rounding can leave u.z above the last cumulative probability; the
  // last candidate takes it. No lobe here reads u.z again: none chooses
  // between reflection and transmission.
#pragma unroll
  for (uint32_t k = 0; k < kGltfLobes; ++k) {
    const float p = c.p[k];
    if (!(p > 0.0f)) continue;
    chosen = k;
    end += p;
    if (u.z < end) break;
  }
  if (chosen == kGltfLobes) return false;
  F3 wi;
  if (chosen == kGltfCoat) {
    const Frame f = make_frame(c.coat_normal);
    const F3 lo = f.to_local(wo);
    if (!(lo.z > 0.0f)) return false;
    const F3 h = sample_ggx_visible_normal(lo, c.coat_alpha, u.x, u.y);
    const float cos_oh = dot(lo, h);
    if (!(cos_oh > 0.0f)) return false;
    const F3 reflected = 2.0f * cos_oh * h - lo;
    if (!(reflected.z > 0.0f)) return false;
    wi = f.to_world(reflected);
  } else {
    if (!(wo.z > 0.0f)) return false;
    if (chosen == kGltfDiffuse) {
      wi = sample_cosine_hemisphere(u.x, u.y);
      if (!(wi.z > 0.0f)) return false;
    } else if (chosen == kGltfSheen) {
      const float sin_theta = sqrtf(fmaxf(1.0f - u.x * u.x, 0.0f));
      float sp, cp;
      lsincos(2.0f * kPi * u.y, sp, cp);
      wi = V(sin_theta * cp, sin_theta * sp, u.x);
      if (!(wi.z > 0.0f)) return false;
    } else {
      const F3 h = sample_ggx_visible_normal(wo, c.alpha, u.x, u.y);
      wi = 2.0f * dot(wo, h) * h - wo;
      if (!(wi.z > 0.0f)) return false;
      if (chosen == kGltfTransmit) wi.z = -wi.z;
    }
    // The base's frame is the shading frame, exactly.
  }
  if (!gltf_scatters_toward(chosen, wi)) return false;
  s.wi = wi;
  s.transmitted = wi.z < 0.0f;
  s.pdf = gltf_pdf(c, wo, wi);
  if (!(s.pdf > 0.0f)) return false;
  s.weight = gltf_evaluate(c, wo, wi) / s.pdf;
  return is_finite(s.weight);
}

}  // namespace lotus
