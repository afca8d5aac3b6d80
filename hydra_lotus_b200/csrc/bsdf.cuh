// SPDX-License-Identifier: Apache-2.0
// UsdPreviewSurface's closure on the device: a Fresnel-attenuated Lambert
// base under a dielectric coat, a GGX reflection lobe, and a share of
// dielectric interface that reflects and transmits
// (backend/vulkan/shaders/bsdf/preview.slang in hydra-lotus). Directions are
// in the shading frame, z along the shading normal on wo's side.
#pragma once

#include "common.cuh"

namespace lotus {

constexpr float kMinAlpha = 1.0e-3f;

struct Closure {
  F3 base_color;
  float alpha;
  float metallic;
  F3 dielectric_f0;
  float dielectric_f90;
  F3 f0;
  float f90;
  float transmission;
  F3 transmission_color;
  float eta;
  bool thin_walled;
  bool smooth;
};

// MakePreviewClosure (preview.slang:60-89).
__device__ __forceinline__ Closure make_closure(F3 base_color, float roughness, float metallic,
    float ior, bool specular_workflow, F3 specular, float transmission, F3 transmission_color,
    bool thin_walled, bool entering) {
  Closure b;
  b.base_color = base_color;
  b.alpha = fmaxf(roughness * roughness, kMinAlpha);
  b.metallic = specular_workflow ? 0.0f : metallic;
  b.transmission = (1.0f - b.metallic) * transmission;
  b.transmission_color = transmission_color;
  b.eta = thin_walled || entering ? ior : 1.0f / ior;
  b.thin_walled = thin_walled;
  b.smooth = roughness * roughness < kMinAlpha || ior == 1.0f;
  if (b.transmission > 0.0f)
    b.metallic = b.transmission < 1.0f ? fminf(b.metallic / (1.0f - b.transmission), 1.0f) : 0.0f;
  const float ratio = 1.0f - 2.0f / (ior + 1.0f);
  b.dielectric_f0 = specular_workflow ? specular : V(ratio * ratio);
  b.dielectric_f90 = specular_workflow || ior > 1.0f ? 1.0f : 0.0f;
  b.f0 = b.base_color * b.metallic + b.dielectric_f0 * (1.0f - b.metallic);
  b.f90 = b.metallic + (1.0f - b.metallic) * b.dielectric_f90;
  return b;
}

__device__ __forceinline__ F3 fresnel_schlick(F3 f0, float f90, float cos_theta) {
  const float weight = lpow5(saturate(1.0f - cos_theta));
  return f0 * (1.0f - weight) + V(f90 * weight);
}

__device__ __forceinline__ F3 dielectric_transmission(const Closure& b, float cos_theta) {
  const F3 fresnel = fresnel_schlick(b.dielectric_f0, b.dielectric_f90, cos_theta);
  return V(1.0f) + fresnel * -1.0f;
}

__device__ __forceinline__ float specular_probability(const Closure& b, F3 wo) {
  if (b.metallic == 1.0f) return 1.0f;
  if (b.dielectric_f90 == 0.0f) return b.metallic;
  const float dielectric = fminf(fmaxf(max_component(fresnel_schlick(
      b.dielectric_f0, b.dielectric_f90, wo.z)), 0.05f), 0.95f);
  return b.metallic + (1.0f - b.metallic) * dielectric;
}

// Exact unpolarized dielectric reflectance (PBR 4th ed., section 9.3).
__device__ __forceinline__ float fresnel_dielectric(float cos_theta, float eta) {
  cos_theta = saturate(cos_theta);
  const float sin2_t = (1.0f - cos_theta * cos_theta) / (eta * eta);
  if (sin2_t >= 1.0f) return 1.0f;
  const float cos_t = sqrtf(1.0f - sin2_t);
  const float parallel = (eta * cos_theta - cos_t) / (eta * cos_theta + cos_t);
  const float perpendicular = (cos_theta - eta * cos_t) / (cos_theta + eta * cos_t);
  return 0.5f * (parallel * parallel + perpendicular * perpendicular);
}

__device__ __forceinline__ float interface_reflectance(const Closure& b, float cos_theta) {
  const float r = fresnel_dielectric(cos_theta, b.eta);
  return b.thin_walled ? 2.0f * r / (1.0f + r) : r;
}

__device__ __forceinline__ float ggx_d(F3 h, float alpha) {
  const float alpha2 = alpha * alpha;
  const float denominator = h.z * h.z * (alpha2 - 1.0f) + 1.0f;
  return alpha2 / (kPi * denominator * denominator);
}

__device__ __forceinline__ float ggx_lambda(F3 w, float alpha) {
  const float tan2 = fmaxf(0.0f, 1.0f - w.z * w.z) / (w.z * w.z);
  return 0.5f * (sqrtf(1.0f + alpha * alpha * tan2) - 1.0f);
}

// Visible-normal sampling by spherical caps (Dupuy and Benyoub 2023).
__device__ __forceinline__ F3 sample_ggx_visible_normal(F3 wo, float alpha, float ux, float uy) {
  const F3 wo_std = normalize(V(wo.x * alpha, wo.y * alpha, wo.z));
  const float phi = 2.0f * kPi * ux;
  const float z = (1.0f - uy) * (1.0f + wo_std.z) - wo_std.z;
  const float sin_theta = sqrtf(saturate(1.0f - z * z));
  float sp, cp;
  lsincos(phi, sp, cp);
  const F3 h_std = V(sin_theta * cp, sin_theta * sp, z) + wo_std;
  return normalize(V(h_std.x * alpha, h_std.y * alpha, h_std.z));
}

__device__ __forceinline__ F3 ggx_eval_cos(const Closure& b, F3 wo, F3 wi) {
  const F3 h = normalize(wo + wi);
  const float g2 = 1.0f / (1.0f + ggx_lambda(wo, b.alpha) + ggx_lambda(wi, b.alpha));
  return fresnel_schlick(b.f0, b.f90, dot(wo, h)) * (ggx_d(h, b.alpha) * g2 / (4.0f * wo.z));
}

__device__ __forceinline__ float ggx_pdf(const Closure& b, F3 wo, F3 wi) {
  const F3 h = normalize(wo + wi);
  const float g1 = 1.0f / (1.0f + ggx_lambda(wo, b.alpha));
  return ggx_d(h, b.alpha) * g1 / (4.0f * wo.z);
}

__device__ __forceinline__ float smith_ratio(const Closure& b, F3 wo, F3 wi) {
  const float lambda_o = ggx_lambda(wo, b.alpha);
  return (1.0f + lambda_o) / (1.0f + lambda_o + ggx_lambda(wi, b.alpha));
}

__device__ __forceinline__ F3 layered_eval_cos(const Closure& b, F3 wo, F3 wi) {
  if (wo.z <= 0.0f || wi.z <= 0.0f) return V(0.0f);
  F3 value = b.base_color * ((1.0f - b.metallic) * wi.z / kPi);
  value = value * dielectric_transmission(b, wo.z) * dielectric_transmission(b, wi.z);
  if (b.f90 > 0.0f) value = value + ggx_eval_cos(b, wo, wi);
  return value;
}

__device__ __forceinline__ float layered_pdf(const Closure& b, F3 wo, F3 wi) {
  if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
  const float specular = specular_probability(b, wo);
  float pdf = (1.0f - specular) * wi.z / kPi;
  if (specular > 0.0f) pdf += specular * ggx_pdf(b, wo, wi);
  return pdf;
}

__device__ __forceinline__ float interface_reflection_eval_cos(const Closure& b, F3 wo, F3 wi) {
  const F3 h = normalize(wo + wi);
  const float g2 = 1.0f / (1.0f + ggx_lambda(wo, b.alpha) + ggx_lambda(wi, b.alpha));
  return interface_reflectance(b, dot(wo, h)) * ggx_d(h, b.alpha) * g2 / (4.0f * wo.z);
}

__device__ __forceinline__ F3 reflection_evaluate(const Closure& b, F3 wo, F3 wi) {
  const F3 layered = layered_eval_cos(b, wo, wi);
  if (b.transmission == 0.0f) return layered;
  F3 value = layered * (1.0f - b.transmission);
  if (!b.smooth && wo.z > 0.0f && wi.z > 0.0f)
    value = value + V(b.transmission * interface_reflection_eval_cos(b, wo, wi));
  return value;
}

__device__ __forceinline__ float reflection_pdf(const Closure& b, F3 wo, F3 wi) {
  const float layered = layered_pdf(b, wo, wi);
  if (b.transmission == 0.0f) return layered;
  float pdf = (1.0f - b.transmission) * layered;
  if (!b.smooth && wo.z > 0.0f && wi.z > 0.0f) {
    const F3 h = normalize(wo + wi);
    pdf += b.transmission * interface_reflectance(b, dot(wo, h)) * ggx_pdf(b, wo, wi);
  }
  return pdf;
}

// The rough interface's transmission value and pdf (preview.slang:267-310).
__device__ __forceinline__ void interface_transmission(const Closure& b, F3 wo, F3 wi,
    float& value, float& pdf) {
  value = 0.0f;
  pdf = 0.0f;
  if (b.transmission == 0.0f || b.smooth || !(wo.z > 0.0f) || !(wi.z < 0.0f)) return;
  if (b.thin_walled) {
    const F3 reflected = V(wi.x, wi.y, -wi.z);
    const F3 h = normalize(wo + reflected);
    const float share = b.transmission * (1.0f - interface_reflectance(b, dot(wo, h)));
    const float g2 = 1.0f / (1.0f + ggx_lambda(wo, b.alpha) + ggx_lambda(reflected, b.alpha));
    value = share * ggx_d(h, b.alpha) * g2 / (4.0f * wo.z);
    pdf = share * ggx_pdf(b, wo, reflected);
    return;
  }
  F3 h = normalize(wo + b.eta * wi);
  if (h.z < 0.0f) h = -h;
  const float cos_oh = dot(wo, h);
  const float cos_ih = dot(wi, h);
  if (!(cos_oh > 0.0f) || !(cos_ih < 0.0f)) return;
  const float denominator = cos_ih + cos_oh / b.eta;
  const float jacobian = -cos_ih / (denominator * denominator);
  const float share = b.transmission * (1.0f - interface_reflectance(b, cos_oh));
  const float d = ggx_d(h, b.alpha);
  const float lambda_o = ggx_lambda(wo, b.alpha);
  const float g1 = 1.0f / (1.0f + lambda_o);
  const float g2 = 1.0f / (1.0f + lambda_o + ggx_lambda(wi, b.alpha));
  pdf = share * (g1 * cos_oh * d / wo.z) * jacobian;
  value = share * (g2 * cos_oh * d / wo.z) * jacobian / (b.eta * b.eta);
}

// BsdfEvaluate: f * |cos(theta_i)| of the non-delta components.
__device__ __forceinline__ F3 bsdf_evaluate(const Closure& b, F3 wo, F3 wi) {
  if (wi.z < 0.0f) {
    float value, pdf;
    interface_transmission(b, wo, wi, value, pdf);
    return b.transmission_color * value;
  }
  return reflection_evaluate(b, wo, wi);
}

// BsdfPdf: the density with which bsdf_sample returns wi as non-delta.
__device__ __forceinline__ float bsdf_pdf(const Closure& b, F3 wo, F3 wi) {
  if (wi.z < 0.0f) {
    float value, pdf;
    interface_transmission(b, wo, wi, value, pdf);
    return pdf;
  }
  return reflection_pdf(b, wo, wi);
}

struct BsdfSample {
  F3 wi;
  F3 weight;
  float pdf;
  bool delta;
  bool transmitted;
};

// SampleInterface (preview.slang:348-405).
__device__ __forceinline__ bool sample_interface(const Closure& b, F3 wo, F3 u, BsdfSample& s) {
  const F3 h = b.smooth ? V(0.0f, 0.0f, 1.0f) : sample_ggx_visible_normal(wo, b.alpha, u.x, u.y);
  const float cos_oh = dot(wo, h);
  if (!(cos_oh > 0.0f)) return false;
  const F3 reflected = 2.0f * cos_oh * h - wo;
  s.delta = b.smooth;
  if (u.z < interface_reflectance(b, cos_oh)) {
    s.wi = reflected;
    if (b.smooth) {
      s.weight = V(1.0f);
      return true;
    }
    if (reflected.z <= 0.0f) return false;
    s.weight = V(smith_ratio(b, wo, reflected));
    s.pdf = reflection_pdf(b, wo, reflected);
    return s.pdf > 0.0f && is_finite(s.weight);
  }
  s.transmitted = true;
  if (b.thin_walled) {
    if (!b.smooth && reflected.z <= 0.0f) return false;
    s.wi = V(reflected.x, reflected.y, -reflected.z);
    s.weight = b.transmission_color * (b.smooth ? 1.0f : smith_ratio(b, wo, reflected));
    if (!b.smooth) {
      float value;
      interface_transmission(b, wo, s.wi, value, s.pdf);
    }
    return is_finite(s.weight);
  }
  const float sin2_t = (1.0f - cos_oh * cos_oh) / (b.eta * b.eta);
  if (sin2_t >= 1.0f) return false;
  const float cos_t = sqrtf(1.0f - sin2_t);
  s.wi = -wo / b.eta + (cos_oh / b.eta - cos_t) * h;
  if (s.wi.z >= 0.0f) return false;
  s.weight = b.transmission_color * ((b.smooth ? 1.0f : smith_ratio(b, wo, s.wi)) / (b.eta * b.eta));
  if (!b.smooth) {
    float value;
    interface_transmission(b, wo, s.wi, value, s.pdf);
  }
  return is_finite(s.weight);
}

// BsdfSample for the preview closure (preview.slang:411-454).
__device__ __forceinline__ bool bsdf_sample(const Closure& b, F3 wo, F3 u, BsdfSample& s) {
  s.wi = V(0.0f);
  s.weight = V(0.0f);
  s.pdf = 0.0f;
  s.delta = false;
  s.transmitted = false;
  if (wo.z <= 0.0f) return false;
  if (b.transmission > 0.0f) {
    if (u.z < b.transmission) return sample_interface(b, wo, V(u.x, u.y, u.z / b.transmission), s);
    u.z = (u.z - b.transmission) / (1.0f - b.transmission);
  }
  if (u.z < specular_probability(b, wo)) {
    const F3 h = sample_ggx_visible_normal(wo, b.alpha, u.x, u.y);
    s.wi = 2.0f * dot(wo, h) * h - wo;
  } else {
    s.wi = sample_cosine_hemisphere(u.x, u.y);
  }
  const float lpdf = layered_pdf(b, wo, s.wi);
  if (!(lpdf > 0.0f)) return false;
  s.pdf = b.transmission > 0.0f ? reflection_pdf(b, wo, s.wi) : lpdf;
  s.weight = layered_eval_cos(b, wo, s.wi) / lpdf;
  if (b.metallic == 1.0f) {
    const F3 h = normalize(wo + s.wi);
    const float lambda_o = ggx_lambda(wo, b.alpha);
    s.weight = fresnel_schlick(b.f0, b.f90, dot(wo, h)) *
        ((1.0f + lambda_o) / (1.0f + lambda_o + ggx_lambda(s.wi, b.alpha)));
  }
  return is_finite(s.weight);
}

}  // namespace lotus
