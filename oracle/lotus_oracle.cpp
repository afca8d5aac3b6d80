// SPDX-License-Identifier: Apache-2.0
//
// TEST INFRASTRUCTURE ONLY: the oracle. A scalar, FP32 CPU restatement of the
// reference's integrator (hydra-lotus v0.9.0), written from its Slang shaders
// and host-side table builders, expression by expression, so that the same
// (pixel, sample index) gives the same path. Each function names the reference
// function it restates. Only tests, the smoke check and the benchmark's CPU
// baseline leg load it, as the checker.
//
// What differs from the reference, and why:
// - Traversal. The reference asks RT hardware for the closest accepted hit
//   (backend/vulkan/shaders/common/scene.slang:424-439). The oracle traverses
//   its own binned-SAH BVH and intersects triangles with the watertight test
//   of Woop, Benthin and Wald (JCGT 2013) in each instance's object space,
//   which is what the CUDA kernels do too. Equal distances resolve to the
//   smaller (instance, primitive), so the closest hit does not depend on the
//   traversal order.
// - Textures. Images (material lookups and the environment) are filtered
//   bilinearly in FP32 (the environment repeating across longitude and
//   clamped at the poles, as the reference's sampler, gpu_scene.cpp:
//   2212-2214), where the reference's sampler hardware uses fixed-point
//   weights.
// - Accumulation. Samples are summed in FP64 (the precision policy), where
//   the reference's image is RGBA32F.
// - The log and power of the glTF closure's albedo axes and sheen are the
//   library's portable ones (restated below), where the reference uses the
//   shading language's; its albedo tables are the library's own cubature
//   of the same lobes (albedo_tables.inc), on the reference's grid.
// Analytic lights (sphere, rect, disk, distant and parallel; their table
// entries, crossing hierarchy, sampling and crossing tests) are restated from
// gpu_scene.cpp:272-610 and scene.slang:680-1178; texture lookups and the
// textured inputs from scene.slang:315-413 and 1184-1260; MaterialX's glTF
// PBR surface, with the general composed closure the reference builds it
// from, from bsdf/albedo.slang, lobes.slang, composed.slang, gltf_pbr.slang
// and scene.slang:1262-1406.

#include "lotus_oracle.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kFloatMax = 3.402823466e+38f;
constexpr uint32_t kNoLights = 0xFFFFFFFFu;
constexpr uint32_t kEnvironmentLight = 0xFFFFFFFFu;
// gpu_scene.hpp:128-172: an analytic light's table entry, its shapes, and
// the crossing hierarchy's child encoding.
constexpr uint32_t kAnalyticLight = 0x80000000u;
constexpr uint32_t kSphereLight = 0, kRectLight = 1, kDiskLight = 2, kDistantLight = 3,
                   kParallelLight = 4;
constexpr uint32_t kLightLeaf = 0x80000000u;
constexpr uint32_t kNoLightChild = 0xFFFFFFFFu;
constexpr uint32_t kLightStackSize = 32;
constexpr uint32_t kRouletteBounces = 3;  // transport.slang:21
constexpr float kMaxSurvival = 0.95f;     // transport.slang:22
constexpr float kMinAlpha = 1.0e-3f;      // preview.slang:17

// ---------------------------------------------------------------------------
// Vectors, with the evaluation order written out.

struct F3 {
  float x, y, z;
};
inline F3 V(float x, float y, float z) { return F3{x, y, z}; }
inline F3 V(float s) { return F3{s, s, s}; }
inline F3 operator+(F3 a, F3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
inline F3 operator-(F3 a, F3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
inline F3 operator-(F3 a) { return V(-a.x, -a.y, -a.z); }
inline F3 operator*(F3 a, F3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
inline F3 operator*(F3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }
inline F3 operator*(float s, F3 a) { return V(s * a.x, s * a.y, s * a.z); }
inline F3 operator/(F3 a, float s) { return V(a.x / s, a.y / s, a.z / s); }
inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 cross(F3 a, F3 b) {
  return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float rsqrt(float x) { return 1.0f / std::sqrt(x); }
inline F3 normalize(F3 a) { return a * rsqrt(dot(a, a)); }
inline float length(F3 a) { return std::sqrt(dot(a, a)); }
inline float saturate(float x) { return std::fmin(std::fmax(x, 0.0f), 1.0f); }
inline float MaxComponent(F3 a) { return std::fmax(a.x, std::fmax(a.y, a.z)); }
inline bool IsFinite(F3 a) {
  return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z);
}
inline float Component(F3 a, int axis) { return axis == 0 ? a.x : axis == 1 ? a.y : a.z; }
inline uint32_t AsUint(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float AsFloat(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

// ---------------------------------------------------------------------------
// Elementary functions. The reference leaves sin, cos, atan2, acos and pow
// to Slang, whose SPIR-V precision is implementation-defined; the CUDA
// kernels use the project's own (Cody-Waite reduction and Taylor
// polynomials, at most 4 ulp from the exact values), and the oracle
// evaluates the same operations in the same order, so both agree bit for
// bit.

inline void lsincos(float x, float& s, float& c) {
  const float k = std::rint(x * 0.636619772f);
  const float r = ((x - k * 1.5703125f) - k * 4.837512969970703e-4f) - k * 7.549790126404332e-8f;
  const float r2 = r * r;
  const float sp = r + r * r2 * (-0.16666667f + r2 * (8.3333338e-3f + r2 * (-1.9841270e-4f +
      r2 * 2.7557319e-6f)));
  const float cp = 1.0f + r2 * (-0.5f + r2 * (4.1666668e-2f + r2 * (-1.3888889e-3f +
      r2 * (2.4801588e-5f + r2 * -2.7557320e-7f))));
  const int q = ((int)k) & 3;
  if (q == 0) {
    s = sp;
    c = cp;
  } else if (q == 1) {
    s = cp;
    c = -sp;
  } else if (q == 2) {
    s = -sp;
    c = -cp;
  } else {
    s = -cp;
    c = sp;
  }
}

inline float lsin(float x) {
  float s, c;
  lsincos(x, s, c);
  return s;
}

inline float lcos(float x) {
  float s, c;
  lsincos(x, s, c);
  return c;
}

// atan(a) for a in [0, 1].
inline float latan_unit(float a) {
  float t = a, base = 0.0f;
  if (a > 0.41421357f) {
    t = (a - 1.0f) / (a + 1.0f);
    base = 0.78539819f;
  }
  const float t2 = t * t;
  const float p = 1.0f + t2 * (-0.33333334f + t2 * (0.2f + t2 * (-0.14285715f + t2 * (0.11111111f +
      t2 * (-0.09090909f + t2 * (0.07692308f + t2 * (-0.06666667f + t2 * (0.05882353f +
      t2 * (-0.05263158f + t2 * 0.04761905f)))))))));
  return base + t * p;
}

inline float latan2(float y, float x) {
  const float ax = std::fabs(x), ay = std::fabs(y);
  const float mx = ax > ay ? ax : ay;
  const float mn = ax > ay ? ay : ax;
  if (mx == 0.0f) return x < 0.0f ? (y < 0.0f ? -3.14159274f : 3.14159274f) : 0.0f;
  float r = latan_unit(mn / mx);
  if (ay > ax) r = 1.57079637f - r;
  if (x < 0.0f) r = 3.14159274f - r;
  return y < 0.0f ? -r : r;
}

// For x in [-1, 1].
inline float lacos(float x) { return latan2(std::sqrt((1.0f - x) * (1.0f + x)), x); }

// pow(x, 5) as products.
inline float lpow5(float x) {
  const float x2 = x * x;
  return x2 * x2 * x;
}


// ---------------------------------------------------------------------------
// sampling.slang

// PcgHash (sampling.slang:9-13).
inline uint32_t PcgHash(uint32_t value) {
  const uint32_t state = value * 747796405u + 2891336453u;
  const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}

// SeedRandom (sampling.slang:16-18).
inline uint32_t SeedRandom(uint32_t pixel_index, uint32_t sample_index) {
  return PcgHash(pixel_index ^ PcgHash(sample_index));
}

// NextRandom (sampling.slang:21-25).
inline float NextRandom(uint32_t& state) {
  state = state * 747796405u + 2891336453u;
  const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return float(((word >> 22u) ^ word) >> 8u) * (1.0f / 16777216.0f);
}

struct ShadingFrame {
  F3 tangent, bitangent, normal;
  F3 ToLocal(F3 d) const { return V(dot(d, tangent), dot(d, bitangent), dot(d, normal)); }
  F3 ToWorld(F3 d) const { return d.x * tangent + d.y * bitangent + d.z * normal; }
};

// MakeShadingFrame (sampling.slang:45-55).
inline ShadingFrame MakeShadingFrame(F3 n) {
  const float sign = n.z >= 0.0f ? 1.0f : -1.0f;
  const float a = -1.0f / (sign + n.z);
  const float b = n.x * n.y * a;
  ShadingFrame f;
  f.tangent = V(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
  f.bitangent = V(b, sign + n.y * n.y * a, -n.y);
  f.normal = n;
  return f;
}

// PowerHeuristic (sampling.slang:67-76).
inline float PowerHeuristic(float chosen, float other) {
  if (!(chosen > 0.0f)) return 0.0f;
  if (std::isinf(chosen)) return std::isinf(other) ? 0.5f : 1.0f;
  const float ratio = other / chosen;
  return 1.0f / (1.0f + ratio * ratio);
}

// SampleCosineHemisphere (sampling.slang:79-84).
inline F3 SampleCosineHemisphere(float ux, float uy) {
  const float radius = std::sqrt(ux);
  const float phi = 2.0f * kPi * uy;
  float s, c;
  lsincos(phi, s, c);
  return V(radius * c, radius * s, std::sqrt(std::fmax(0.0f, 1.0f - ux)));
}

// ---------------------------------------------------------------------------
// bsdf/preview.slang

struct PreviewClosure {
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
PreviewClosure MakePreviewClosure(F3 base_color, float roughness, float metallic,
    float ior, bool specular_workflow, F3 specular, float transmission,
    F3 transmission_color, bool thin_walled, bool entering) {
  PreviewClosure b;
  b.base_color = base_color;
  b.alpha = std::fmax(roughness * roughness, kMinAlpha);
  b.metallic = specular_workflow ? 0.0f : metallic;
  b.transmission = (1.0f - b.metallic) * transmission;
  b.transmission_color = transmission_color;
  b.eta = thin_walled || entering ? ior : 1.0f / ior;
  b.thin_walled = thin_walled;
  b.smooth = roughness * roughness < kMinAlpha || ior == 1.0f;
  if (b.transmission > 0.0f) {
    b.metallic = b.transmission < 1.0f
        ? std::fmin(b.metallic / (1.0f - b.transmission), 1.0f)
        : 0.0f;
  }
  const float ratio = 1.0f - 2.0f / (ior + 1.0f);
  b.dielectric_f0 = specular_workflow ? specular : V(ratio * ratio);
  b.dielectric_f90 = specular_workflow || ior > 1.0f ? 1.0f : 0.0f;
  b.f0 = b.base_color * b.metallic + b.dielectric_f0 * (1.0f - b.metallic);
  b.f90 = b.metallic + (1.0f - b.metallic) * b.dielectric_f90;
  return b;
}

// FresnelSchlick (preview.slang:92-95).
inline F3 FresnelSchlick(F3 f0, float f90, float cos_theta) {
  const float weight = lpow5(saturate(1.0f - cos_theta));
  return f0 * (1.0f - weight) + V(f90 * weight);
}

// DielectricTransmission (preview.slang:100-104).
inline F3 DielectricTransmission(const PreviewClosure& b, float cos_theta) {
  const F3 fresnel = FresnelSchlick(b.dielectric_f0, b.dielectric_f90, cos_theta);
  return V(1.0f) + fresnel * -1.0f;
}

// SpecularProbability (preview.slang:106-112).
inline float SpecularProbability(const PreviewClosure& b, F3 wo) {
  if (b.metallic == 1.0f) return 1.0f;
  if (b.dielectric_f90 == 0.0f) return b.metallic;
  const float dielectric = std::fmin(std::fmax(MaxComponent(FresnelSchlick(
      b.dielectric_f0, b.dielectric_f90, wo.z)), 0.05f), 0.95f);
  return b.metallic + (1.0f - b.metallic) * dielectric;
}

// FresnelDielectric (preview.slang:118-127).
inline float FresnelDielectric(float cos_theta, float eta) {
  cos_theta = saturate(cos_theta);
  const float sin2_t = (1.0f - cos_theta * cos_theta) / (eta * eta);
  if (sin2_t >= 1.0f) return 1.0f;
  const float cos_t = std::sqrt(1.0f - sin2_t);
  const float parallel = (eta * cos_theta - cos_t) / (eta * cos_theta + cos_t);
  const float perpendicular = (cos_theta - eta * cos_t) / (cos_theta + eta * cos_t);
  return 0.5f * (parallel * parallel + perpendicular * perpendicular);
}

// InterfaceReflectance (preview.slang:132-135).
inline float InterfaceReflectance(const PreviewClosure& b, float cos_theta) {
  const float r = FresnelDielectric(cos_theta, b.eta);
  return b.thin_walled ? 2.0f * r / (1.0f + r) : r;
}

// GgxD (preview.slang:138-142).
inline float GgxD(F3 h, float alpha) {
  const float alpha2 = alpha * alpha;
  const float denominator = h.z * h.z * (alpha2 - 1.0f) + 1.0f;
  return alpha2 / (kPi * denominator * denominator);
}

// GgxLambda (preview.slang:145-148).
inline float GgxLambda(F3 w, float alpha) {
  const float tan2 = std::fmax(0.0f, 1.0f - w.z * w.z) / (w.z * w.z);
  return 0.5f * (std::sqrt(1.0f + alpha * alpha * tan2) - 1.0f);
}

// SampleGgxVisibleNormal (preview.slang:152-160).
inline F3 SampleGgxVisibleNormal(F3 wo, float alpha, float ux, float uy) {
  const F3 wo_std = normalize(V(wo.x * alpha, wo.y * alpha, wo.z));
  const float phi = 2.0f * kPi * ux;
  const float z = (1.0f - uy) * (1.0f + wo_std.z) - wo_std.z;
  const float sin_theta = std::sqrt(saturate(1.0f - z * z));
  float sp, cp;
  lsincos(phi, sp, cp);
  const F3 h_std = V(sin_theta * cp, sin_theta * sp, z) + wo_std;
  return normalize(V(h_std.x * alpha, h_std.y * alpha, h_std.z));
}

// GgxEvalCos (preview.slang:164-170).
inline F3 GgxEvalCos(const PreviewClosure& b, F3 wo, F3 wi) {
  const F3 h = normalize(wo + wi);
  const float g2 = 1.0f / (1.0f + GgxLambda(wo, b.alpha) + GgxLambda(wi, b.alpha));
  return FresnelSchlick(b.f0, b.f90, dot(wo, h)) *
         (GgxD(h, b.alpha) * g2 / (4.0f * wo.z));
}

// GgxPdf (preview.slang:173-177).
inline float GgxPdf(const PreviewClosure& b, F3 wo, F3 wi) {
  const F3 h = normalize(wo + wi);
  const float g1 = 1.0f / (1.0f + GgxLambda(wo, b.alpha));
  return GgxD(h, b.alpha) * g1 / (4.0f * wo.z);
}

// SmithRatio (preview.slang:180-183).
inline float SmithRatio(const PreviewClosure& b, F3 wo, F3 wi) {
  const float lambda_o = GgxLambda(wo, b.alpha);
  return (1.0f + lambda_o) / (1.0f + lambda_o + GgxLambda(wi, b.alpha));
}

// LayeredEvalCos (preview.slang:187-198).
F3 LayeredEvalCos(const PreviewClosure& b, F3 wo, F3 wi) {
  if (wo.z <= 0.0f || wi.z <= 0.0f) return V(0.0f);
  F3 value = b.base_color * ((1.0f - b.metallic) * wi.z / kPi);
  value = value * DielectricTransmission(b, wo.z) * DielectricTransmission(b, wi.z);
  if (b.f90 > 0.0f) value = value + GgxEvalCos(b, wo, wi);
  return value;
}

// LayeredPdf (preview.slang:202-212).
float LayeredPdf(const PreviewClosure& b, F3 wo, F3 wi) {
  if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
  const float specular = SpecularProbability(b, wo);
  float pdf = (1.0f - specular) * wi.z / kPi;
  if (specular > 0.0f) pdf += specular * GgxPdf(b, wo, wi);
  return pdf;
}

// InterfaceReflectionEvalCos (preview.slang:216-222).
float InterfaceReflectionEvalCos(const PreviewClosure& b, F3 wo, F3 wi) {
  const F3 h = normalize(wo + wi);
  const float g2 = 1.0f / (1.0f + GgxLambda(wo, b.alpha) + GgxLambda(wi, b.alpha));
  return InterfaceReflectance(b, dot(wo, h)) * GgxD(h, b.alpha) * g2 / (4.0f * wo.z);
}

// PreviewReflectionEvaluate (preview.slang:227-238).
F3 PreviewReflectionEvaluate(const PreviewClosure& b, F3 wo, F3 wi) {
  const F3 layered = LayeredEvalCos(b, wo, wi);
  if (b.transmission == 0.0f) return layered;
  F3 value = layered * (1.0f - b.transmission);
  if (!b.smooth && wo.z > 0.0f && wi.z > 0.0f)
    value = value + V(b.transmission * InterfaceReflectionEvalCos(b, wo, wi));
  return value;
}

// PreviewReflectionPdf (preview.slang:240-252).
float PreviewReflectionPdf(const PreviewClosure& b, F3 wo, F3 wi) {
  const float layered = LayeredPdf(b, wo, wi);
  if (b.transmission == 0.0f) return layered;
  float pdf = (1.0f - b.transmission) * layered;
  if (!b.smooth && wo.z > 0.0f && wi.z > 0.0f) {
    const F3 h = normalize(wo + wi);
    pdf += b.transmission * InterfaceReflectance(b, dot(wo, h)) * GgxPdf(b, wo, wi);
  }
  return pdf;
}

struct InterfaceTransmission {
  float value;
  float pdf;
};

// PreviewTransmission (preview.slang:267-310).
InterfaceTransmission PreviewTransmission(const PreviewClosure& b, F3 wo, F3 wi) {
  InterfaceTransmission r{0.0f, 0.0f};
  if (b.transmission == 0.0f || b.smooth || !(wo.z > 0.0f) || !(wi.z < 0.0f)) return r;
  if (b.thin_walled) {
    const F3 reflected = V(wi.x, wi.y, -wi.z);
    const F3 h = normalize(wo + reflected);
    const float share = b.transmission * (1.0f - InterfaceReflectance(b, dot(wo, h)));
    const float g2 = 1.0f / (1.0f + GgxLambda(wo, b.alpha) + GgxLambda(reflected, b.alpha));
    r.value = share * GgxD(h, b.alpha) * g2 / (4.0f * wo.z);
    r.pdf = share * GgxPdf(b, wo, reflected);
    return r;
  }
  F3 h = normalize(wo + b.eta * wi);
  if (h.z < 0.0f) h = -h;
  const float cos_oh = dot(wo, h);
  const float cos_ih = dot(wi, h);
  if (!(cos_oh > 0.0f) || !(cos_ih < 0.0f)) return r;
  const float denominator = cos_ih + cos_oh / b.eta;
  const float jacobian = -cos_ih / (denominator * denominator);
  const float share = b.transmission * (1.0f - InterfaceReflectance(b, cos_oh));
  const float d = GgxD(h, b.alpha);
  const float lambda_o = GgxLambda(wo, b.alpha);
  const float g1 = 1.0f / (1.0f + lambda_o);
  const float g2 = 1.0f / (1.0f + lambda_o + GgxLambda(wi, b.alpha));
  r.pdf = share * (g1 * cos_oh * d / wo.z) * jacobian;
  r.value = share * (g2 * cos_oh * d / wo.z) * jacobian / (b.eta * b.eta);
  return r;
}

// PreviewEvaluate (preview.slang:314-319).
F3 PreviewEvaluate(const PreviewClosure& b, F3 wo, F3 wi) {
  if (wi.z < 0.0f) return b.transmission_color * PreviewTransmission(b, wo, wi).value;
  return PreviewReflectionEvaluate(b, wo, wi);
}

// PreviewPdf (preview.slang:322-327).
float PreviewPdf(const PreviewClosure& b, F3 wo, F3 wi) {
  if (wi.z < 0.0f) return PreviewTransmission(b, wo, wi).pdf;
  return PreviewReflectionPdf(b, wo, wi);
}

struct BsdfSampleResult {
  F3 wi;
  F3 weight;
  float pdf;
  bool delta;
  bool transmitted;
};

// SampleInterface (preview.slang:348-405).
bool SampleInterface(const PreviewClosure& b, F3 wo, F3 u, BsdfSampleResult& s) {
  const F3 h = b.smooth ? V(0.0f, 0.0f, 1.0f) : SampleGgxVisibleNormal(wo, b.alpha, u.x, u.y);
  const float cos_oh = dot(wo, h);
  if (!(cos_oh > 0.0f)) return false;
  const F3 reflected = 2.0f * cos_oh * h - wo;
  s.delta = b.smooth;
  if (u.z < InterfaceReflectance(b, cos_oh)) {
    s.wi = reflected;
    if (b.smooth) {
      s.weight = V(1.0f);
      return true;
    }
    if (reflected.z <= 0.0f) return false;
    s.weight = V(SmithRatio(b, wo, reflected));
    s.pdf = PreviewReflectionPdf(b, wo, reflected);
    return s.pdf > 0.0f && IsFinite(s.weight);
  }
  s.transmitted = true;
  if (b.thin_walled) {
    if (!b.smooth && reflected.z <= 0.0f) return false;
    s.wi = V(reflected.x, reflected.y, -reflected.z);
    s.weight = b.transmission_color * (b.smooth ? 1.0f : SmithRatio(b, wo, reflected));
    if (!b.smooth) s.pdf = PreviewTransmission(b, wo, s.wi).pdf;
    return IsFinite(s.weight);
  }
  const float sin2_t = (1.0f - cos_oh * cos_oh) / (b.eta * b.eta);
  if (sin2_t >= 1.0f) return false;
  const float cos_t = std::sqrt(1.0f - sin2_t);
  s.wi = -wo / b.eta + (cos_oh / b.eta - cos_t) * h;
  if (s.wi.z >= 0.0f) return false;
  s.weight = b.transmission_color *
      ((b.smooth ? 1.0f : SmithRatio(b, wo, s.wi)) / (b.eta * b.eta));
  if (!b.smooth) s.pdf = PreviewTransmission(b, wo, s.wi).pdf;
  return IsFinite(s.weight);
}

// PreviewSample (preview.slang:411-454).
bool PreviewSample(const PreviewClosure& b, F3 wo, F3 u, BsdfSampleResult& s) {
  s.wi = V(0.0f);
  s.weight = V(0.0f);
  s.pdf = 0.0f;
  s.delta = false;
  s.transmitted = false;
  if (wo.z <= 0.0f) return false;
  if (b.transmission > 0.0f) {
    if (u.z < b.transmission)
      return SampleInterface(b, wo, V(u.x, u.y, u.z / b.transmission), s);
    u.z = (u.z - b.transmission) / (1.0f - b.transmission);
  }
  if (u.z < SpecularProbability(b, wo)) {
    const F3 h = SampleGgxVisibleNormal(wo, b.alpha, u.x, u.y);
    s.wi = 2.0f * dot(wo, h) * h - wo;
  } else {
    s.wi = SampleCosineHemisphere(u.x, u.y);
  }
  const float layered_pdf = LayeredPdf(b, wo, s.wi);
  if (!(layered_pdf > 0.0f)) return false;
  s.pdf = b.transmission > 0.0f ? PreviewReflectionPdf(b, wo, s.wi) : layered_pdf;
  s.weight = LayeredEvalCos(b, wo, s.wi) / layered_pdf;
  if (b.metallic == 1.0f) {
    const F3 h = normalize(wo + s.wi);
    const float lambda_o = GgxLambda(wo, b.alpha);
    s.weight = FresnelSchlick(b.f0, b.f90, dot(wo, h)) *
        ((1.0f + lambda_o) / (1.0f + lambda_o + GgxLambda(s.wi, b.alpha)));
  }
  return IsFinite(s.weight);
}

// ---------------------------------------------------------------------------
// Composed closures and MaterialX's glTF PBR surface (bsdf/albedo.slang,
// bsdf/lobes.slang, bsdf/composed.slang, bsdf/gltf_pbr.slang), with the
// scene passes' configuration: no attenuating layer and no dielectric
// refraction, thin-wall or delta paths (LOTUS_COMPOSED_FULL 0).

// The elementary functions the albedo axes and the sheen need, written out
// as the library does (natural log by 2 atanh((m - 1) / (m + 1)) after
// splitting off the binary exponent; exp by Cody and Waite's reduction and
// Taylor's series), so that host and device agree bit for bit where the
// reference uses the shading language's log and pow.
inline float LLog(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? -AsFloat(0x7f800000u) : AsFloat(0x7fc00000u);
  int e = 0;
  if (x < 1.17549435e-38f) {
    x *= 8388608.0f;
    e = -23;
  }
  const uint32_t b = AsUint(x);
  e += (int)((b >> 23) & 0xffu) - 127;
  float m = AsFloat((b & 0x7fffffu) | 0x3f800000u);
  if (m > 1.41421354f) {
    m *= 0.5f;
    e += 1;
  }
  const float s = (m - 1.0f) / (m + 1.0f);
  const float s2 = s * s;
  const float p = s2 * (0.333333343f + s2 * (0.2f + s2 * (0.142857149f + s2 * (0.111111112f +
      s2 * (0.0909090936f + s2 * (0.0769230798f + s2 * 0.0666666701f))))));
  const float log_m = 2.0f * s + 2.0f * s * p;
  const float fe = (float)e;
  return fe * 0.693145751953125f + (fe * 1.42860677e-6f + log_m);
}

inline float LExp(float x) {
  if (!(x > -104.0f)) return x == x ? 0.0f : x;
  if (x > 89.0f) return AsFloat(0x7f800000u);
  const float k = std::rint(x * 1.44269502f);
  const float r = (x - k * 0.693145751953125f) - k * 1.42860677e-6f;
  const float p = 1.0f + r * (1.0f + r * (0.5f + r * (0.166666672f + r * (0.0416666679f +
      r * (0.00833333377f + r * (0.00138888892f + r * (0.000198412701f + r * 2.48015876e-5f)))))));
  int ki = (int)k;
  float scale = 1.0f;
  if (ki < -126) {
    ki += 64;
    scale = 5.42101086e-20f;
  } else if (ki > 127) {
    ki -= 1;
    scale = 2.0f;
  }
  return p * AsFloat((uint32_t)(ki + 127) << 23) * scale;
}

inline float LPow(float x, float y) { return x > 0.0f ? LExp(y * LLog(x)) : 0.0f; }

// The directional albedo tables' data: the library's own generated tables
// (albedo.slang's layout, 76800 floats).
const float kAlbedoTableData[] = {
#include "../hydra_lotus_b200/csrc/albedo_tables.inc"
};
static_assert(sizeof(kAlbedoTableData) == 76800 * sizeof(float), "albedo tables");

// albedo.slang:22-65.
constexpr uint32_t kAlbedoGgx = 0, kAlbedoSchlickShare = 1, kAlbedoDielectric = 2, kAlbedoSheen = 3;
constexpr uint32_t kDielectricEntering = 0, kDielectricLeaving = 1, kDielectricThin = 2,
                   kDielectricSheets = 3;
constexpr uint32_t kGgxCosines = 32, kDielectricCosines = 48, kAlbedoAlphas = 32, kAlbedoIndices = 16;
constexpr float kAlbedoMinIndex = 1.01f, kAlbedoMaxIndex = 3.0f;
constexpr float kMinCosine = 2.0e-4f, kCosineSlope = 4.0f, kAlphaSlope = 2.0f, kIndexSlope = 0.5f;
constexpr float kMinSheenAxis = 0.005f;
constexpr uint32_t kCriticalNode = kDielectricCosines / 2;
constexpr float kCriticalCoordinate = float(kCriticalNode) / float(kDielectricCosines - 1);
constexpr float kMinEvanescent = 2.0e-3f;

uint32_t AlbedoTableOffset(uint32_t table) {
  const uint32_t ggx = kGgxCosines * kAlbedoAlphas;
  if (table <= kAlbedoDielectric) return table * ggx;
  return (table - 1) * ggx + kDielectricSheets * kAlbedoIndices * kDielectricCosines * kAlbedoAlphas;
}

// albedo.slang:86-190.
inline float LogLinearScale(float v, float slope) { return LLog(v) + slope * v; }

inline float LogLinearCoordinate(float v, float low, float high, float slope) {
  const float clamped = std::fmin(std::fmax(v, low), high);
  return (LogLinearScale(clamped, slope) - LogLinearScale(low, slope)) /
      (LogLinearScale(high, slope) - LogLinearScale(low, slope));
}

inline float CosineCoordinate(float c) { return LogLinearCoordinate(c, kMinCosine, 1.0f, kCosineSlope); }
inline float AlphaCoordinate(float a) { return LogLinearCoordinate(a, kMinAlpha, 1.0f, kAlphaSlope); }
inline float SheenCoordinate(float r) { return LogLinearCoordinate(r, kMinSheenAxis, 1.0f, kAlphaSlope); }
inline float IndexCoordinate(float index) {
  return LogLinearCoordinate(index - 1.0f, kAlbedoMinIndex - 1.0f, kAlbedoMaxIndex - 1.0f, kIndexSlope);
}

inline float CriticalCosine(float index) { return std::sqrt(std::fmax(1.0f - 1.0f / (index * index), 0.0f)); }

inline float EvanescentScale(float mu, float index, float critical) {
  const float tau = std::fmax(index * std::sqrt(std::fmax(critical * critical - mu * mu, 0.0f)),
      kMinEvanescent);
  return LLog(mu) - LLog(tau) + kCosineSlope * mu;
}

inline float LeavingCoordinate(float cos_theta, float index) {
  const float critical = CriticalCosine(index);
  if (cos_theta < critical) {
    const float low = EvanescentScale(kMinCosine, index, critical);
    const float high = EvanescentScale(critical, index, critical);
    return kCriticalCoordinate *
        saturate((EvanescentScale(std::fmax(cos_theta, kMinCosine), index, critical) - low) / (high - low));
  }
  const float refracted = std::sqrt(std::fmax(1.0f - index * index * (1.0f - cos_theta * cos_theta), 0.0f));
  // lerp(kCriticalCoordinate, 1, x)
  const float x = CosineCoordinate(refracted);
  return kCriticalCoordinate + (1.0f - kCriticalCoordinate) * x;
}

// albedo.slang:246-312.
inline void CubicWeights(float t, float w[4]) {
  const float t2 = t * t;
  const float t3 = t2 * t;
  w[0] = -0.5f * t3 + t2 - 0.5f * t;
  w[1] = 1.5f * t3 - 2.5f * t2 + 1.0f;
  w[2] = -1.5f * t3 + 2.0f * t2 + 0.5f * t;
  w[3] = 0.5f * t3 - 0.5f * t2;
}

float FetchNode(uint32_t base, uint32_t cosines, int cosine, int alpha, int first, int last) {
  const int last_alpha = (int)kAlbedoAlphas - 1;
  const int c = std::min(std::max(cosine, first), last);
  const int a = std::min(std::max(alpha, 0), last_alpha);
  const int dc = cosine < first ? 1 : (cosine > last ? -1 : 0);
  const int da = alpha < 0 ? 1 : (alpha > last_alpha ? -1 : 0);
  const float at = kAlbedoTableData[base + (uint32_t)(a * (int)cosines + c)];
  if (dc == 0 && da == 0) return at;
  const float inner = kAlbedoTableData[base + (uint32_t)((a + da) * (int)cosines + c + dc)];
  return 2.0f * at - inner;
}

float FetchSlice(uint32_t base, uint32_t cosines, float x_cosine, float x_alpha, bool split) {
  const float fc = saturate(x_cosine) * float(cosines - 1);
  const float fa = saturate(x_alpha) * float(kAlbedoAlphas - 1);
  const int c0 = (int)std::min((uint32_t)fc, cosines - 2);
  const int a0 = (int)std::min((uint32_t)fa, kAlbedoAlphas - 2);
  int first = 0;
  int last = (int)cosines - 1;
  if (split) {
    if (c0 < (int)kCriticalNode) last = (int)kCriticalNode;
    else first = (int)kCriticalNode;
  }
  float wc[4], wa[4];
  CubicWeights(fc - float(c0), wc);
  CubicWeights(fa - float(a0), wa);
  float value = 0.0f;
  for (int j = 0; j < 4; ++j) {
    float row = 0.0f;
    for (int i = 0; i < 4; ++i) row += wc[i] * FetchNode(base, cosines, c0 + i - 1, a0 + j - 1, first, last);
    value += wa[j] * row;
  }
  return value;
}

// albedo.slang:314-373.
float AlbedoGgx(float cos_theta, float alpha) {
  return FetchSlice(AlbedoTableOffset(kAlbedoGgx), kGgxCosines, CosineCoordinate(cos_theta),
      AlphaCoordinate(alpha), false);
}

float AlbedoSchlickShare(float cos_theta, float alpha) {
  return FetchSlice(AlbedoTableOffset(kAlbedoSchlickShare), kGgxCosines, CosineCoordinate(cos_theta),
      AlphaCoordinate(alpha), false);
}

float AlbedoSheen(float cos_theta, float roughness) {
  return std::fmax(FetchSlice(AlbedoTableOffset(kAlbedoSheen), kGgxCosines, CosineCoordinate(cos_theta),
      SheenCoordinate(roughness), false), 0.0f);
}

float AlbedoDielectric(float cos_theta, float alpha, float eta, bool thin_walled) {
  uint32_t sheet = thin_walled ? kDielectricThin : kDielectricEntering;
  float index = eta;
  if (eta < 1.0f) {
    index = 1.0f / eta;
    sheet = thin_walled ? kDielectricThin : kDielectricLeaving;
  }
  index = std::fmin(std::fmax(index, kAlbedoMinIndex), kAlbedoMaxIndex);
  const float fi = IndexCoordinate(index) * float(kAlbedoIndices - 1);
  const int i0 = (int)std::min((uint32_t)fi, kAlbedoIndices - 2);
  const bool split = sheet == kDielectricLeaving;
  const float x_cosine = split ? LeavingCoordinate(cos_theta, index) : CosineCoordinate(cos_theta);
  const float x_alpha = AlphaCoordinate(alpha);
  const uint32_t slice_size = kDielectricCosines * kAlbedoAlphas;
  const uint32_t base = AlbedoTableOffset(kAlbedoDielectric) + sheet * kAlbedoIndices * slice_size;
  float slices[4];
  for (int j = 0; j < 4; ++j) {
    const int slice = std::min(std::max(i0 + j - 1, 0), (int)kAlbedoIndices - 1);
    slices[j] = FetchSlice(base + (uint32_t)slice * slice_size, kDielectricCosines, x_cosine, x_alpha, split);
  }
  if (i0 == 0) slices[0] = 2.0f * slices[1] - slices[2];
  if (i0 == (int)kAlbedoIndices - 2) slices[3] = 2.0f * slices[2] - slices[1];
  float w[4];
  CubicWeights(fi - float(i0), w);
  return w[0] * slices[0] + w[1] * slices[1] + w[2] * slices[2] + w[3] * slices[3];
}

// --- Lobes (lobes.slang) ---------------------------------------------------

constexpr uint32_t kLambertLobe = 0, kGgxSchlickLobe = 1, kGgxDielectricLobe = 2, kSheenLobe = 3;
constexpr uint32_t kScatterReflect = 1, kScatterTransmit = 2, kScatterBoth = 3;
constexpr float kMinSheenRoughness = 0.005f;

struct Lobe {
  uint32_t type;
  F3 normal;
  F3 color;
  F3 f90;
  float alpha;
  float eta;
  uint32_t scatter;
  bool thin_walled;
  bool transmit;
  bool smooth;
  bool compensate;
  F3 compensation;
};

Lobe MakeLobe(uint32_t type, F3 normal) {
  Lobe lobe;
  lobe.type = type;
  lobe.normal = normal;
  lobe.color = V(1.0f);
  lobe.f90 = V(1.0f);
  lobe.alpha = 1.0f;
  lobe.eta = 1.0f;
  lobe.scatter = kScatterReflect;
  lobe.thin_walled = false;
  lobe.transmit = false;
  lobe.smooth = false;
  lobe.compensate = false;
  lobe.compensation = V(1.0f);
  return lobe;
}

Lobe MakeLambertLobe(F3 color, F3 normal) {
  Lobe lobe = MakeLobe(kLambertLobe, normal);
  lobe.color = color;
  return lobe;
}

Lobe MakeGgxSchlickLobe(F3 f0, F3 f90, float alpha, F3 normal, bool compensate) {
  Lobe lobe = MakeLobe(kGgxSchlickLobe, normal);
  lobe.color = f0;
  lobe.f90 = f90;
  lobe.alpha = std::fmax(alpha, kMinAlpha);
  lobe.compensate = compensate;
  return lobe;
}

Lobe MakeSheenLobe(F3 color, float roughness, F3 normal) {
  Lobe lobe = MakeLobe(kSheenLobe, normal);
  lobe.color = color;
  lobe.alpha = std::fmax(roughness, kMinSheenRoughness);
  return lobe;
}

Lobe MakeGgxDielectricLobe(float eta, F3 tint, float alpha, uint32_t scatter, bool thin_walled, F3 normal,
    bool compensate) {
  Lobe lobe = MakeLobe(kGgxDielectricLobe, normal);
  lobe.color = tint;
  lobe.alpha = std::fmax(alpha, kMinAlpha);
  lobe.eta = eta;
  lobe.scatter = scatter;
  lobe.thin_walled = thin_walled;
  lobe.smooth = alpha < kMinAlpha || eta == 1.0f;
  lobe.compensate = compensate;
  return lobe;
}

inline bool LobeScattersToward(const Lobe& lobe, F3 wi) {
  if (lobe.type == kGgxDielectricLobe)
    return wi.z > 0.0f ? (lobe.scatter & kScatterReflect) != 0 : (lobe.scatter & kScatterTransmit) != 0;
  return lobe.transmit ? wi.z < 0.0f : wi.z > 0.0f;
}

inline F3 SchlickFresnel(F3 f0, F3 f90, float cos_theta) {
  const float weight = lpow5(saturate(1.0f - cos_theta));
  return f0 * (1.0f - weight) + f90 * weight;
}

inline float DielectricReflectance(const Lobe& lobe, float cos_theta) {
  const float r = FresnelDielectric(cos_theta, lobe.eta);
  return lobe.thin_walled ? 2.0f * r / (1.0f + r) : r;
}

inline float GgxReflection(F3 wo, F3 wi, F3 h, float alpha) {
  const float g2 = 1.0f / (1.0f + GgxLambda(wo, alpha) + GgxLambda(wi, alpha));
  return GgxD(h, alpha) * g2 / (4.0f * wo.z);
}

inline float GgxReflectionPdf(F3 wo, F3 h, float alpha) {
  const float g1 = 1.0f / (1.0f + GgxLambda(wo, alpha));
  return GgxD(h, alpha) * g1 / (4.0f * wo.z);
}

// SheenValue (lobes.slang:260-271).
F3 SheenValue(const Lobe& lobe, F3 wo, F3 wi) {
  if (!(wi.z > 0.0f)) return V(0.0f);
  const F3 h = normalize(wo + wi);
  const float inverse = 1.0f / lobe.alpha;
  const float sin2 = std::fmax(1.0f - h.z * h.z, 0.0f);
  const float d = (2.0f + inverse) * LPow(sin2, 0.5f * inverse) / (2.0f * kPi);
  return lobe.color * lobe.compensation * (d * wi.z / (4.0f * (wi.z + wo.z - wi.z * wo.z)));
}

// DielectricValue (lobes.slang:273-303), reflection only.
F3 DielectricValue(const Lobe& lobe, F3 wo, F3 wi) {
  if (lobe.smooth) return V(0.0f);
  if (wi.z > 0.0f) {
    if ((lobe.scatter & kScatterReflect) == 0) return V(0.0f);
    const F3 h = normalize(wo + wi);
    return lobe.color * lobe.compensation *
        (DielectricReflectance(lobe, dot(wo, h)) * GgxReflection(wo, wi, h, lobe.alpha));
  }
  return V(0.0f);
}

// LobeValue (lobes.slang:306-325).
F3 LobeValue(const Lobe& lobe, F3 wo, F3 wi) {
  if (!(wo.z > 0.0f)) return V(0.0f);
  switch (lobe.type) {
    case kLambertLobe:
      return wi.z > 0.0f ? lobe.color * (wi.z / kPi) : V(0.0f);
    case kGgxSchlickLobe: {
      const F3 wr = lobe.transmit ? V(wi.x, wi.y, -wi.z) : wi;
      if (!(wr.z > 0.0f)) return V(0.0f);
      const F3 h = normalize(wo + wr);
      return SchlickFresnel(lobe.color, lobe.f90, dot(wo, h)) * lobe.compensation *
          GgxReflection(wo, wr, h, lobe.alpha);
    }
    case kSheenLobe:
      return SheenValue(lobe, wo, wi);
    default:
      return DielectricValue(lobe, wo, wi);
  }
}

// DielectricPdf (lobes.slang:327-362), reflection only.
float DielectricPdf(const Lobe& lobe, F3 wo, F3 wi) {
  if (lobe.smooth) return 0.0f;
  const bool both = lobe.scatter == kScatterBoth;
  if (wi.z > 0.0f) {
    if ((lobe.scatter & kScatterReflect) == 0) return 0.0f;
    const F3 h = normalize(wo + wi);
    const float choice = both ? DielectricReflectance(lobe, dot(wo, h)) : 1.0f;
    return choice * GgxReflectionPdf(wo, h, lobe.alpha);
  }
  return 0.0f;
}

// LobePdf (lobes.slang:364-383).
float LobePdf(const Lobe& lobe, F3 wo, F3 wi) {
  if (!(wo.z > 0.0f)) return 0.0f;
  switch (lobe.type) {
    case kLambertLobe:
      return wi.z > 0.0f ? wi.z / kPi : 0.0f;
    case kGgxSchlickLobe: {
      const F3 wr = lobe.transmit ? V(wi.x, wi.y, -wi.z) : wi;
      return wr.z > 0.0f ? GgxReflectionPdf(wo, normalize(wo + wr), lobe.alpha) : 0.0f;
    }
    case kSheenLobe:
      return wi.z > 0.0f ? 1.0f / (2.0f * kPi) : 0.0f;
    default:
      return DielectricPdf(lobe, wo, wi);
  }
}

// LobeSample (lobes.slang:446-508), without the dielectric's refraction,
// thin-wall and delta paths.
bool LobeSample(const Lobe& lobe, F3 wo, F3 u, F3& wi) {
  wi = V(0.0f, 0.0f, 1.0f);
  if (!(wo.z > 0.0f)) return false;
  switch (lobe.type) {
    case kLambertLobe:
      wi = SampleCosineHemisphere(u.x, u.y);
      return wi.z > 0.0f;
    case kGgxSchlickLobe: {
      const F3 h = SampleGgxVisibleNormal(wo, lobe.alpha, u.x, u.y);
      wi = 2.0f * dot(wo, h) * h - wo;
      if (!(wi.z > 0.0f)) return false;
      if (lobe.transmit) wi.z = -wi.z;
      return true;
    }
    case kSheenLobe: {
      const float sin_theta = std::sqrt(std::fmax(1.0f - u.x * u.x, 0.0f));
      const float phi = 2.0f * kPi * u.y;
      float s, c;
      lsincos(phi, s, c);
      wi = V(sin_theta * c, sin_theta * s, u.x);
      return wi.z > 0.0f;
    }
    default: {
      const F3 h = SampleGgxVisibleNormal(wo, lobe.alpha, u.x, u.y);
      const float cos_oh = dot(wo, h);
      if (!(cos_oh > 0.0f)) return false;
      const F3 reflected = 2.0f * cos_oh * h - wo;
      bool reflect = lobe.scatter == kScatterReflect;
      if (lobe.scatter == kScatterBoth) reflect = u.z < DielectricReflectance(lobe, cos_oh);
      if (reflect) {
        wi = reflected;
        return reflected.z > 0.0f;
      }
      return false;
    }
  }
}

// --- Composed closures (composed.slang) -------------------------------------

constexpr uint32_t kMaxLobes = 6;
constexpr float kSelectionFloor = 0.05f;

struct ComposedClosure {
  uint32_t count = 0;
  Lobe lobes[kMaxLobes];
  F3 weights[kMaxLobes];
  float probabilities[kMaxLobes];
};

struct ComposedBuilder {
  ComposedClosure closure;
  F3 albedos[kMaxLobes];
  F3 estimates[kMaxLobes];
};

// No layer of these closures attenuates (ComposedAttenuate is never
// called): every attenuation factor is 1.
inline F3 AttenuationFactor() { return V(1.0f); }

ComposedBuilder ComposedBegin() {
  ComposedBuilder builder;
  builder.closure.count = 0;
  for (uint32_t k = 0; k < kMaxLobes; ++k) {
    builder.closure.lobes[k] = MakeLambertLobe(V(0.0f), V(0.0f, 0.0f, 1.0f));
    builder.closure.weights[k] = V(0.0f);
    builder.closure.probabilities[k] = 0.0f;
    builder.albedos[k] = V(0.0f);
    builder.estimates[k] = V(0.0f);
  }
  return builder;
}

uint32_t ComposedPush(ComposedBuilder& b, const Lobe& lobe, F3 albedo, F3 estimate) {
  const uint32_t k = b.closure.count;
  if (k >= kMaxLobes) return k;
  b.closure.count = k + 1;
  b.closure.weights[k] = V(1.0f);
  b.closure.lobes[k] = lobe;
  b.albedos[k] = albedo;
  b.estimates[k] = estimate;
  return k;
}

uint32_t ComposedAddLambert(ComposedBuilder& b, const Lobe& lobe, F3 wo) {
  const F3 albedo = dot(wo, lobe.normal) > 0.0f ? lobe.color : V(0.0f);
  return ComposedPush(b, lobe, albedo, albedo);
}

uint32_t ComposedAddSchlick(ComposedBuilder& b, const Lobe& added, F3 wo, float e1, float share) {
  Lobe lobe = added;
  F3 albedo = V(0.0f);
  if (dot(wo, lobe.normal) > 0.0f) {
    if (lobe.compensate && e1 > 0.0f) lobe.compensation = V(1.0f) + lobe.color * ((1.0f - e1) / e1);
    albedo = (lobe.color * (e1 - share) + lobe.f90 * share) * lobe.compensation;
  }
  return ComposedPush(b, lobe, lobe.transmit ? V(0.0f) : albedo, albedo);
}

uint32_t ComposedAddWeighted(ComposedBuilder& b, const Lobe& lobe, F3 weight, F3 albedo) {
  const uint32_t k = ComposedPush(b, lobe, albedo, albedo * lobe.color);
  if (k < kMaxLobes) b.closure.weights[k] = weight;
  return k;
}

void ComposedScale(ComposedBuilder& b, uint32_t begin, uint32_t end, F3 scale) {
  for (uint32_t k = begin; k < std::min(end, b.closure.count); ++k)
    b.closure.weights[k] = b.closure.weights[k] * scale;
}

void ComposedMix(ComposedBuilder& b, uint32_t begin, uint32_t split, uint32_t end, float mix) {
  ComposedScale(b, begin, split, V(1.0f - mix));
  ComposedScale(b, split, end, V(mix));
}

F3 ComposedAlbedo(const ComposedBuilder& b, uint32_t begin, uint32_t end) {
  F3 albedo = V(0.0f);
  for (uint32_t k = begin; k < std::min(end, b.closure.count); ++k)
    albedo = albedo + b.closure.weights[k] * AttenuationFactor() * b.albedos[k];
  return albedo;
}

inline F3 SaturateRgb(F3 v) { return V(saturate(v.x), saturate(v.y), saturate(v.z)); }

void ComposedLayer(ComposedBuilder& b, uint32_t begin, uint32_t split, uint32_t end) {
  const F3 top = ComposedAlbedo(b, begin, split);
  ComposedScale(b, split, end, SaturateRgb(V(1.0f) - top));
}

void ComposedLayerScalar(ComposedBuilder& b, uint32_t begin, uint32_t split, uint32_t end) {
  const F3 top = ComposedAlbedo(b, begin, split);
  ComposedScale(b, split, end, SaturateRgb(V(1.0f - MaxComponent(top))));
}

ComposedClosure ComposedFinalize(const ComposedBuilder& b) {
  ComposedClosure closure = b.closure;
  float total = 0.0f;
  for (uint32_t k = 0; k < closure.count; ++k) {
    const float estimate = MaxComponent(closure.weights[k] * AttenuationFactor() * b.estimates[k]);
    closure.probabilities[k] = estimate > 0.0f ? estimate : 0.0f;
    total += closure.probabilities[k];
  }
  if (!(total > 0.0f)) return closure;
  float floored = 0.0f;
  for (uint32_t k = 0; k < closure.count; ++k)
    if (closure.probabilities[k] > 0.0f) {
      closure.probabilities[k] = std::fmax(closure.probabilities[k] / total, kSelectionFloor);
      floored += closure.probabilities[k];
    }
  for (uint32_t k = 0; k < closure.count; ++k) closure.probabilities[k] /= floored;
  return closure;
}

F3 ComposedEvaluate(const ComposedClosure& c, F3 wo, F3 wi) {
  F3 value = V(0.0f);
  for (uint32_t k = 0; k < c.count; ++k) {
    const Lobe& lobe = c.lobes[k];
    if (!LobeScattersToward(lobe, wi)) continue;
    const ShadingFrame frame = MakeShadingFrame(lobe.normal);
    value = value + c.weights[k] * AttenuationFactor() * LobeValue(lobe, frame.ToLocal(wo), frame.ToLocal(wi));
  }
  return value;
}

float ComposedPdf(const ComposedClosure& c, F3 wo, F3 wi) {
  float pdf = 0.0f;
  for (uint32_t k = 0; k < c.count; ++k) {
    const Lobe& lobe = c.lobes[k];
    if (!(c.probabilities[k] > 0.0f) || !LobeScattersToward(lobe, wi)) continue;
    const ShadingFrame frame = MakeShadingFrame(lobe.normal);
    pdf += c.probabilities[k] * LobePdf(lobe, frame.ToLocal(wo), frame.ToLocal(wi));
  }
  return pdf;
}

bool ComposedSample(const ComposedClosure& c, F3 wo, F3 u, BsdfSampleResult& s) {
  s.wi = V(0.0f, 0.0f, 1.0f);
  s.weight = V(0.0f);
  s.pdf = 0.0f;
  s.delta = false;
  s.transmitted = false;
  uint32_t chosen = kMaxLobes;
  float start = 0.0f, end = 0.0f;
  for (uint32_t k = 0; k < c.count; ++k) {
    const float p = c.probabilities[k];
    if (!(p > 0.0f)) continue;
    chosen = k;
    start = end;
    end += p;
    if (u.z < end) break;
  }
  if (chosen == kMaxLobes) return false;
  const float probability = c.probabilities[chosen];
  u.z = std::fmin(std::fmax((u.z - start) / probability, 0.0f), 0.99999994f);
  const Lobe& lobe = c.lobes[chosen];
  const ShadingFrame frame = MakeShadingFrame(lobe.normal);
  F3 local;
  if (!LobeSample(lobe, frame.ToLocal(wo), u, local)) return false;
  s.wi = frame.ToWorld(local);
  if (!LobeScattersToward(lobe, s.wi)) return false;
  s.transmitted = s.wi.z < 0.0f;
  s.pdf = ComposedPdf(c, wo, s.wi);
  if (!(s.pdf > 0.0f)) return false;
  s.weight = ComposedEvaluate(c, wo, s.wi) / s.pdf;
  return IsFinite(s.weight);
}

// --- MaterialX's glTF PBR (gltf_pbr.slang) ------------------------------------

constexpr float kGltfClearcoatIndex = 1.5f;

struct GltfPbrInputs {
  F3 base_color;
  float roughness;
  float metallic;
  float dielectric_f0;
  float specular;
  F3 specular_color;
  float transmission;
  float clearcoat;
  float clearcoat_roughness;
  F3 clearcoat_normal;
  F3 sheen_color;
  float sheen_roughness;
};

// MakeGltfPbrInputs (gltf_pbr.slang:54-72).
GltfPbrInputs MakeGltfPbrInputs(F3 base_color, float roughness, float metallic) {
  GltfPbrInputs in;
  in.base_color = base_color;
  in.roughness = roughness;
  in.metallic = metallic;
  in.dielectric_f0 = 0.04f;
  in.specular = 1.0f;
  in.specular_color = V(1.0f);
  in.transmission = 0.0f;
  in.clearcoat = 0.0f;
  in.clearcoat_roughness = 0.0f;
  in.clearcoat_normal = V(0.0f, 0.0f, 1.0f);
  in.sheen_color = V(0.0f);
  in.sheen_roughness = 0.0f;
  return in;
}

struct GltfPbrTerms {
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
GltfPbrTerms MakeGltfPbrTerms(const GltfPbrInputs& in, F3 wo) {
  GltfPbrTerms t;
  t.base_color = in.base_color;
  t.alpha = std::fmax(in.roughness * in.roughness, kMinAlpha);
  t.metallic = in.metallic;
  t.e1 = 0.0f;
  t.share = 0.0f;
  if (wo.z > 0.0f) {
    t.e1 = AlbedoGgx(wo.z, t.alpha);
    t.share = AlbedoSchlickShare(wo.z, t.alpha);
  }
  t.f0 = SaturateRgb(in.specular_color * in.dielectric_f0) * in.specular;
  t.f90 = in.specular;
  t.transmission = in.transmission;
  t.coat_scale = 0.0f;
  t.coat_dim = 0.0f;
  t.coat_alpha = std::fmax(in.clearcoat_roughness * in.clearcoat_roughness, kMinAlpha);
  t.coat_normal = in.clearcoat_normal.z > 0.0f ? in.clearcoat_normal : V(0.0f, 0.0f, 1.0f);
  const float coat_cos = dot(wo, t.coat_normal);
  if (in.clearcoat > 0.0f && coat_cos > 0.0f) {
    const float reflected = AlbedoDielectric(coat_cos, t.coat_alpha, kGltfClearcoatIndex, false);
    const float coat_e1 = AlbedoGgx(coat_cos, t.coat_alpha);
    const float coat_root = (1.0f - kGltfClearcoatIndex) / (1.0f + kGltfClearcoatIndex);
    float compensation = 1.0f;
    if (coat_e1 > 0.0f) compensation += coat_root * coat_root * (1.0f - coat_e1) / coat_e1;
    t.coat_scale = in.clearcoat * compensation;
    t.coat_dim = saturate(t.coat_scale * reflected);
  }
  t.sheen_color = in.sheen_color;
  t.sheen_roughness = std::fmax(in.sheen_roughness * in.sheen_roughness, kMinSheenRoughness);
  t.sheen_dim = 0.0f;
  const float sheen = MaxComponent(in.sheen_color);
  if (sheen > 0.0f && wo.z > 0.0f) {
    const float e = AlbedoSheen(wo.z, t.sheen_roughness);
    if (e > 1.0f) t.sheen_color = in.sheen_color * (1.0f / e);
    t.sheen_dim = saturate(sheen * std::fmin(e, 1.0f));
  }
  return t;
}

// MakeGltfPbrClosure (gltf_pbr.slang:230-290).
ComposedClosure MakeGltfPbrClosure(const GltfPbrTerms& t, F3 wo) {
  const F3 normal = V(0.0f, 0.0f, 1.0f);
  const F3 white = V(1.0f);
  ComposedBuilder b = ComposedBegin();
  const uint32_t coat = b.closure.count;
  if (t.coat_scale > 0.0f)
    ComposedAddWeighted(b,
        MakeGgxDielectricLobe(kGltfClearcoatIndex, white, t.coat_alpha, kScatterReflect, false, t.coat_normal,
            false),
        V(t.coat_scale), V(t.coat_dim / t.coat_scale));
  const uint32_t sheen = b.closure.count;
  if (t.sheen_dim > 0.0f)
    ComposedAddWeighted(b, MakeSheenLobe(white, t.sheen_roughness, normal), t.sheen_color,
        V(t.sheen_dim / MaxComponent(t.sheen_color)));
  const bool dielectric = t.metallic < 1.0f;
  const uint32_t top = b.closure.count;
  if (dielectric && t.f90 > 0.0f)
    ComposedAddSchlick(b, MakeGgxSchlickLobe(t.f0, V(t.f90), t.alpha, normal, true), wo, t.e1, t.share);
  const uint32_t diffuse = b.closure.count;
  if (dielectric && t.transmission < 1.0f) ComposedAddLambert(b, MakeLambertLobe(t.base_color, normal), wo);
  const uint32_t transmitted = b.closure.count;
  if (dielectric && t.transmission > 0.0f) {
    Lobe lobe = MakeGgxSchlickLobe(white, white, t.alpha, normal, true);
    lobe.transmit = true;
    const uint32_t k = ComposedAddSchlick(b, lobe, wo, t.e1, t.share);
    ComposedScale(b, k, k + 1, t.base_color);
  }
  const uint32_t metal = b.closure.count;
  if (t.transmission > 0.0f) ComposedMix(b, diffuse, transmitted, metal, t.transmission);
  ComposedLayerScalar(b, top, diffuse, metal);
  if (t.metallic > 0.0f)
    ComposedAddSchlick(b, MakeGgxSchlickLobe(t.base_color, white, t.alpha, normal, true), wo, t.e1, t.share);
  const uint32_t end = b.closure.count;
  ComposedMix(b, top, metal, end, t.metallic);
  ComposedLayerScalar(b, sheen, top, end);
  ComposedLayer(b, coat, sheen, end);
  return ComposedFinalize(b);
}


// ---------------------------------------------------------------------------
// Scene

struct Box {
  float lo[3] = {kFloatMax, kFloatMax, kFloatMax};
  float hi[3] = {-kFloatMax, -kFloatMax, -kFloatMax};
  void Grow(const float* p) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], p[a]);
      hi[a] = std::max(hi[a], p[a]);
    }
  }
  void Grow(const Box& b) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], b.lo[a]);
      hi[a] = std::max(hi[a], b.hi[a]);
    }
  }
  float Area() const {
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    if (!(dx >= 0.0f)) return 0.0f;
    return 2.0f * (dx * dy + dy * dz + dz * dx);
  }
};

// A binary BVH over boxes, built top-down with binned SAH. Leaves hold up
// to four primitives from `order`.
struct Bvh {
  struct Node {
    Box box;
    uint32_t left = 0;   // interior: left child; right child is left + 1
    uint32_t first = 0;  // leaf: first index into order
    uint32_t count = 0;  // leaf: primitive count; 0 for an interior node
  };
  std::vector<Node> nodes;
  std::vector<uint32_t> order;

  void Build(const std::vector<Box>& boxes) {
    const uint32_t n = static_cast<uint32_t>(boxes.size());
    order.resize(n);
    for (uint32_t i = 0; i < n; ++i) order[i] = i;
    nodes.clear();
    nodes.reserve(n > 0 ? 2 * n : 1);
    nodes.emplace_back();
    if (n == 0) return;
    std::vector<float> centroids(3 * size_t{n});
    for (uint32_t i = 0; i < n; ++i)
      for (int a = 0; a < 3; ++a)
        centroids[3 * i + a] = 0.5f * (boxes[i].lo[a] + boxes[i].hi[a]);
    struct Task { uint32_t node, first, count; };
    std::vector<Task> stack{{0, 0, n}};
    while (!stack.empty()) {
      const Task t = stack.back();
      stack.pop_back();
      Node& node = nodes[t.node];
      Box bounds, cbounds;
      for (uint32_t i = t.first; i < t.first + t.count; ++i) {
        bounds.Grow(boxes[order[i]]);
        cbounds.Grow(&centroids[3 * order[i]]);
      }
      node.box = bounds;
      if (t.count <= 4) {
        node.first = t.first;
        node.count = t.count;
        continue;
      }
      constexpr int kBins = 16;
      float best_cost = std::numeric_limits<float>::infinity();
      int best_axis = -1, best_split = 0;
      for (int a = 0; a < 3; ++a) {
        const float extent = cbounds.hi[a] - cbounds.lo[a];
        if (!(extent > 0.0f)) continue;
        Box bin_box[kBins];
        uint32_t bin_count[kBins] = {};
        for (uint32_t i = t.first; i < t.first + t.count; ++i) {
          int b = static_cast<int>((centroids[3 * order[i] + a] - cbounds.lo[a]) / extent * kBins);
          b = std::min(std::max(b, 0), kBins - 1);
          bin_box[b].Grow(boxes[order[i]]);
          ++bin_count[b];
        }
        float right_area[kBins];
        uint32_t right_count[kBins];
        Box acc;
        uint32_t cnt = 0;
        for (int b = kBins - 1; b > 0; --b) {
          acc.Grow(bin_box[b]);
          cnt += bin_count[b];
          right_area[b] = acc.Area();
          right_count[b] = cnt;
        }
        acc = Box();
        cnt = 0;
        for (int b = 0; b < kBins - 1; ++b) {
          acc.Grow(bin_box[b]);
          cnt += bin_count[b];
          if (cnt == 0 || right_count[b + 1] == 0) continue;
          const float cost = acc.Area() * cnt + right_area[b + 1] * right_count[b + 1];
          if (cost < best_cost) {
            best_cost = cost;
            best_axis = a;
            best_split = b;
          }
        }
      }
      uint32_t mid;
      if (best_axis < 0) {
        mid = t.first + t.count / 2;  // coincident centroids: split the list
      } else {
        const int a = best_axis;
        const float extent = cbounds.hi[a] - cbounds.lo[a];
        auto it = std::partition(order.begin() + t.first, order.begin() + t.first + t.count,
            [&](uint32_t p) {
              int b = static_cast<int>((centroids[3 * p + a] - cbounds.lo[a]) / extent * kBins);
              b = std::min(std::max(b, 0), kBins - 1);
              return b <= best_split;
            });
        mid = static_cast<uint32_t>(it - order.begin());
        if (mid == t.first || mid == t.first + t.count) mid = t.first + t.count / 2;
      }
      const uint32_t left = static_cast<uint32_t>(nodes.size());
      nodes.emplace_back();
      nodes.emplace_back();
      nodes[t.node].left = left;
      nodes[t.node].count = 0;
      stack.push_back({left, t.first, mid - t.first});
      stack.push_back({left + 1, mid, t.first + t.count - mid});
    }
  }
};

struct Geometry {
  std::vector<F3> positions;
  std::vector<uint32_t> triangles;
  std::vector<F3> normals;  // 3 per triangle, or empty
  std::vector<float> texcoords;  // set k, triangle i, corner c: 6 * (k * triangles + i) + 2 * c
  uint32_t texcoord_sets = 0;
  // Colour sets: each one RGB per triangle corner, or one for the mesh.
  std::vector<std::vector<F3>> colors;
  Bvh bvh;
};

struct Instance {
  float m[16];   // world_from_object, column-major
  float inv[12]; // object_from_world, rows of a 3x4 matrix
  uint32_t geometry;
  uint32_t material;
  uint32_t texcoord_set;  // lotus_instance::texcoord_set (0: none)
  uint32_t color_set;     // lotus_instance::color_set (0: none)
  Box world;
};

// A texture decoded to linear RGBA floats, rows from the top.
struct Texture {
  uint32_t width = 0, height = 0;
  std::vector<float> rgba;
};

struct LightRecord {
  float pdf;
  float threshold;
  uint32_t alias;
  uint32_t instance;
};

// GpuAnalyticLightRecord (gpu_scene.hpp:144-166).
struct AnalyticLight {
  float position[4];
  float axis_u[4];
  float axis_v[4];
  float normal[4];
  float radiance[4];
  uint32_t shape;
};

// GpuLightNode (gpu_scene.hpp:174-186): per child its bounds, the child's
// bits in low.w.
struct LightNode {
  float low0[4], high0[4], low1[4], high1[4];
};

struct Environment {
  bool bound = false;
  uint32_t width = 0, height = 0;
  std::vector<float> texels;  // RGBA
  F3 scale{1, 1, 1};
  F3 rows[3];                 // environment_from_world
  uint32_t columns = 0, rows_count = 0;
  std::vector<float> floats;  // density, marginal, conditional
  double mean = 0.0;
};

}  // namespace

struct oracle_scene {
  std::vector<Geometry> geometries;
  std::vector<Instance> instances;
  std::vector<lotus_material> materials;
  Bvh tlas;
  std::vector<LightRecord> lights;
  std::vector<uint32_t> light_offsets;
  std::vector<lotus_light> light_inputs;
  std::vector<AnalyticLight> analytic;
  std::vector<LightNode> light_nodes;
  std::vector<uint32_t> distant;
  float environment_selection = 0.0f;
  F3 environment_constant{0, 0, 0};
  Environment env;
  std::vector<Texture> textures;
  std::vector<lotus_texture_input> inputs;
};

namespace {

// Object-from-world as a 3x4 float matrix, by Gauss-Jordan elimination in
// double of the affine part.
bool InvertAffine(const float* m, float* inv) {
  double a[3][4];
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) a[r][c] = m[c * 4 + r];
    a[r][3] = m[12 + r];
  }
  // [A | t] -> inverse [A^-1 | -A^-1 t]
  double aug[3][6];
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) aug[r][c] = a[r][c];
    for (int c = 0; c < 3; ++c) aug[r][3 + c] = r == c ? 1.0 : 0.0;
  }
  for (int c = 0; c < 3; ++c) {
    int p = c;
    for (int r = c + 1; r < 3; ++r)
      if (std::fabs(aug[r][c]) > std::fabs(aug[p][c])) p = r;
    if (aug[p][c] == 0.0) return false;
    for (int k = 0; k < 6; ++k) std::swap(aug[c][k], aug[p][k]);
    const double s = aug[c][c];
    for (int k = 0; k < 6; ++k) aug[c][k] /= s;
    for (int r = 0; r < 3; ++r) {
      if (r == c) continue;
      const double f = aug[r][c];
      for (int k = 0; k < 6; ++k) aug[r][k] -= f * aug[c][k];
    }
  }
  for (int r = 0; r < 3; ++r) {
    double t = 0.0;
    for (int c = 0; c < 3; ++c) {
      inv[r * 4 + c] = static_cast<float>(aug[r][3 + c]);
      t -= aug[r][3 + c] * a[c][3];
    }
    inv[r * 4 + 3] = static_cast<float>(t);
  }
  return true;
}

// mul(world_from_object, float4(p, 1)).xyz
inline F3 TransformPoint(const float* m, F3 p) {
  return V(m[0] * p.x + m[4] * p.y + m[8] * p.z + m[12],
           m[1] * p.x + m[5] * p.y + m[9] * p.z + m[13],
           m[2] * p.x + m[6] * p.y + m[10] * p.z + m[14]);
}

// EmissionEstimate (gpu_scene.cpp:144-180): its
// constant emission, or a lookup's bound for texels in [0, 1] (its
// fallback when the lookup names no image).
double EmissionEstimate(const oracle_scene& s, const lotus_material& m) {
  double e[3];
  const uint32_t lookup = m.lookups[LOTUS_SLOT_EMISSION];
  for (int c = 0; c < 3; ++c) {
    if (lookup == LOTUS_NO_LOOKUP) {
      e[c] = m.emission[c];
    } else {
      const lotus_texture_input& in = s.inputs[lookup - 1];
      e[c] = in.texture == LOTUS_NO_TEXTURE ? std::max(0.0f, in.fallback[c])
                                           : double{std::max(0.0f, in.scale[c])} + std::max(0.0f, in.bias[c]);
    }
  }
  // glTF PBR's emissive (slot 5, as UsdPreviewSurface's emission) is
  // scaled by its strength.
  const double factor = m.model == LOTUS_MODEL_GLTF_PBR ? double{m.emissive_strength} : 1.0;
  const double mean = factor * (e[0] + e[1] + e[2]) / 3.0;
  return std::isfinite(mean) && mean > 0.0 ? mean : 0.0;
}

// WorldTriangleArea (gpu_scene.cpp:182-203).
double WorldTriangleArea(const Geometry& g, uint32_t t, const float* m) {
  double corners[3][3];
  for (int k = 0; k < 3; ++k) {
    const F3 p = g.positions[g.triangles[3 * t + k]];
    for (int r = 0; r < 3; ++r)
      corners[k][r] = double{m[r]} * p.x + double{m[4 + r]} * p.y +
                      double{m[8 + r]} * p.z + m[12 + r];
  }
  double a[3], b[3];
  for (int r = 0; r < 3; ++r) {
    a[r] = corners[1][r] - corners[0][r];
    b[r] = corners[2][r] - corners[0][r];
  }
  const double x = a[1] * b[2] - a[2] * b[1];
  const double y = a[2] * b[0] - a[0] * b[2];
  const double z = a[0] * b[1] - a[1] * b[0];
  const double area = 0.5 * std::sqrt(x * x + y * y + z * z);
  return std::isfinite(area) ? area : 0.0;
}

// SceneRadius (gpu_scene.cpp:233-270).
double SceneRadius(const oracle_scene& s) {
  constexpr double kInf = std::numeric_limits<double>::infinity();
  std::vector<std::array<double, 6>> object(s.geometries.size());
  std::vector<bool> done(s.geometries.size(), false);
  std::array<double, 6> world{kInf, kInf, kInf, -kInf, -kInf, -kInf};
  for (const Instance& inst : s.instances) {
    auto& b = object[inst.geometry];
    if (!done[inst.geometry]) {
      done[inst.geometry] = true;
      b = {kInf, kInf, kInf, -kInf, -kInf, -kInf};
      for (const F3& p : s.geometries[inst.geometry].positions) {
        const double v[3] = {p.x, p.y, p.z};
        for (int a = 0; a < 3; ++a) {
          b[a] = std::min(b[a], v[a]);
          b[3 + a] = std::max(b[3 + a], v[a]);
        }
      }
    }
    if (!(b[0] <= b[3])) continue;
    const float* m = inst.m;
    for (int corner = 0; corner < 8; ++corner) {
      const double p[3] = {b[(corner & 1) ? 3 : 0], b[(corner & 2) ? 4 : 1], b[(corner & 4) ? 5 : 2]};
      for (int r = 0; r < 3; ++r) {
        const double v = m[r] * p[0] + m[4 + r] * p[1] + m[8 + r] * p[2] + m[12 + r];
        world[r] = std::min(world[r], v);
        world[3 + r] = std::max(world[3 + r], v);
      }
    }
  }
  if (!(world[0] <= world[3])) return 0.0;
  const double d[3] = {world[3] - world[0], world[4] - world[1], world[5] - world[2]};
  const double radius = 0.5 * std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  return std::isfinite(radius) ? radius : 0.0;
}

// BuildEnvironmentDistribution (gpu_scene.cpp:638-711), RGBA32F texels.
void BuildEnvironmentDistribution(Environment& env) {
  constexpr double kPiD = 3.14159265358979323846;
  const uint32_t columns = std::min(env.width, 2048u);
  const uint32_t rows = std::min(env.height, 1024u);
  env.columns = columns;
  env.rows_count = rows;
  const size_t cells = size_t{columns} * rows;
  std::vector<double> sums(cells, 0.0);
  std::vector<uint32_t> counts(cells, 0);
  const double scale[3] = {env.scale.x, env.scale.y, env.scale.z};
  for (uint32_t y = 0; y < env.height; ++y) {
    const size_t row = uint64_t{y} * rows / env.height;
    for (uint32_t x = 0; x < env.width; ++x) {
      const size_t column = uint64_t{x} * columns / env.width;
      const float* t = &env.texels[4 * (size_t{y} * env.width + x)];
      double radiance = 0.0;
      for (int c = 0; c < 3; ++c) radiance += std::max(double{t[c]}, 0.0) * scale[c];
      sums[row * columns + column] += radiance / 3.0;
      ++counts[row * columns + column];
    }
  }
  std::vector<double> values(cells), row_sums(rows, 0.0);
  double total = 0.0;
  for (uint32_t row = 0; row < rows; ++row) {
    const double sin_theta = std::sin(kPiD * (row + 0.5) / rows);
    for (uint32_t column = 0; column < columns; ++column) {
      const size_t cell = size_t{row} * columns + column;
      values[cell] = sums[cell] / counts[cell] * sin_theta;
      row_sums[row] += values[cell];
    }
    total += row_sums[row];
  }
  const double mean = total / static_cast<double>(cells);
  std::vector<float> density(cells, 0.0f), marginal(rows + 1, 0.0f),
      conditional(size_t{rows} * (columns + 1), 0.0f);
  env.mean = 0.0;
  if (mean > 0.0 && std::isfinite(mean)) {
    env.mean = mean;
    for (size_t cell = 0; cell < cells; ++cell)
      density[cell] = static_cast<float>(values[cell] / mean);
    double cumulative = 0.0;
    for (uint32_t row = 0; row < rows; ++row) {
      cumulative += row_sums[row];
      marginal[row + 1] = static_cast<float>(cumulative / total);
      float* cdf = conditional.data() + size_t{row} * (columns + 1);
      double along = 0.0;
      for (uint32_t column = 0; column < columns; ++column) {
        along += values[size_t{row} * columns + column];
        cdf[column + 1] = row_sums[row] > 0.0
            ? static_cast<float>(along / row_sums[row])
            : static_cast<float>(column + 1) / columns;
      }
      cdf[columns] = 1.0f;
    }
    marginal[rows] = 1.0f;
  }
  env.floats.clear();
  env.floats.insert(env.floats.end(), density.begin(), density.end());
  env.floats.insert(env.floats.end(), marginal.begin(), marginal.end());
  env.floats.insert(env.floats.end(), conditional.begin(), conditional.end());
  env.bound = env.mean > 0.0;
}

struct D3 {
  double x, y, z;
};
inline D3 Column(const float* m, int c) { return D3{m[4 * c], m[4 * c + 1], m[4 * c + 2]}; }
inline double Dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline D3 Cross(D3 a, D3 b) {
  return D3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline D3 Scale(D3 a, double s) { return D3{a.x * s, a.y * s, a.z * s}; }
inline void Store(float* out, D3 v, double w) {
  out[0] = static_cast<float>(v.x);
  out[1] = static_cast<float>(v.y);
  out[2] = static_cast<float>(v.z);
  out[3] = static_cast<float>(w);
}

// MakeAnalyticLight (gpu_scene.cpp:272-369): the record and its table
// weight, the estimated power over 2 pi (a distant light's through a disk
// of the scene's radius). False for a light that emits nothing.
bool MakeAnalyticLight(const lotus_light& light, double scene_radius, double& weight, AnalyticLight& record) {
  constexpr double kPiD = 3.14159265358979323846;
  const float* m = light.world_from_light;
  const D3 x = Column(m, 0), y = Column(m, 1), z = Column(m, 2), origin = Column(m, 3);
  const double determinant = Dot(x, Cross(y, z));
  record = AnalyticLight{};
  double extent = 0.0, scale = 1.0;
  if (light.shape == LOTUS_LIGHT_SPHERE) {
    const double radius = light.radius * std::cbrt(std::fabs(determinant));
    extent = 4.0 * kPiD * radius * radius;
    record.shape = kSphereLight;
    Store(record.position, origin, radius);
    Store(record.normal, D3{0, 0, 0}, extent);
  } else if (light.shape == LOTUS_LIGHT_RECT || light.shape == LOTUS_LIGHT_DISK) {
    const bool rect = light.shape == LOTUS_LIGHT_RECT;
    const D3 u = Scale(x, rect ? 0.5 * light.width : light.radius);
    const D3 v = Scale(y, rect ? 0.5 * light.height : light.radius);
    const D3 normal = Cross(u, v);
    const double length = std::sqrt(Dot(normal, normal));
    extent = (rect ? 4.0 : kPiD) * length;
    record.shape = rect ? kRectLight : kDiskLight;
    Store(record.position, origin, 0.0);
    Store(record.axis_u, u, 0.0);
    Store(record.axis_v, v, 0.0);
    if (length > 0.0) Store(record.normal, Scale(normal, (determinant < 0.0 ? 1.0 : -1.0) / length), extent);
  } else {
    const double length = std::sqrt(Dot(z, z));
    if (!(length > 0.0)) return false;
    const double theta = std::min(static_cast<double>(light.angle) * kPiD / 360.0, kPiD);
    const double half = std::sin(0.5 * theta);
    const double one_minus_cos = 2.0 * half * half;
    const double sin2 = std::sin(theta) * std::sin(theta);
    Store(record.axis_u, Scale(z, 1.0 / length), one_minus_cos);
    record.shape = kParallelLight;
    extent = 1.0;
    if (theta > 0.0) {
      extent = theta <= 0.5 * kPiD ? kPiD * sin2 : kPiD;
      if (light.normalize) scale = 1.0 / (theta <= 0.5 * kPiD ? kPiD * sin2 : (2.0 - sin2) * kPiD);
      if (static_cast<float>(one_minus_cos) >= std::numeric_limits<float>::min()) {
        record.shape = kDistantLight;
      } else {
        scale *= extent;
        extent = 1.0;
      }
    }
  }
  if (light.normalize && light.shape != LOTUS_LIGHT_DISTANT) scale = 1.0 / extent;
  double radiance[3];
  for (int c = 0; c < 3; ++c) radiance[c] = light.radiance[c] * scale;
  const double mean = (radiance[0] + radiance[1] + radiance[2]) / 3.0;
  if (!(extent > 0.0) || !std::isfinite(extent) || !(mean > 0.0) ||
      !(radiance[0] <= std::numeric_limits<float>::max() && radiance[1] <= std::numeric_limits<float>::max() &&
          radiance[2] <= std::numeric_limits<float>::max()))
    return false;
  Store(record.radiance, D3{radiance[0], radiance[1], radiance[2]}, 0.0);
  weight = mean * extent / 2.0;
  if (light.shape == LOTUS_LIGHT_DISTANT) weight *= scene_radius * scene_radius;
  if (!std::isfinite(weight)) weight = std::numeric_limits<double>::max();
  return true;
}

// A bounded light's box (BoundLight, gpu_scene.cpp:398-428): its extent
// widened by 1e-4 of itself plus 1e-5 of the coordinates' magnitude, then
// rounded outwards.
struct LightBounds {
  float low[3], high[3];
  double centre[3];
  uint32_t index;
};

LightBounds BoundLight(const AnalyticLight& light, uint32_t index) {
  LightBounds b;
  b.index = index;
  for (int a = 0; a < 3; ++a) {
    const double centre = light.position[a];
    const double u = light.axis_u[a], v = light.axis_v[a];
    const double extent = light.shape == kSphereLight ? light.position[3]
        : light.shape == kRectLight                   ? std::fabs(u) + std::fabs(v)
                                                      : std::sqrt(u * u + v * v);
    const double margin = 1e-4 * extent + 1e-5 * (std::fabs(centre) + extent);
    b.centre[a] = centre;
    b.low[a] = std::nextafter(static_cast<float>(centre - extent - margin), -std::numeric_limits<float>::infinity());
    b.high[a] = std::nextafter(static_cast<float>(centre + extent + margin), std::numeric_limits<float>::infinity());
  }
  return b;
}

void StoreBounds(float* low, float* high, const LightBounds* first, const LightBounds* last, uint32_t child) {
  for (int a = 0; a < 3; ++a) {
    low[a] = std::numeric_limits<float>::max();
    high[a] = -std::numeric_limits<float>::max();
    for (const LightBounds* it = first; it != last; ++it) {
      low[a] = std::min(low[a], it->low[a]);
      high[a] = std::max(high[a], it->high[a]);
    }
  }
  std::memcpy(&low[3], &child, 4);
}

// BuildLightNode (gpu_scene.cpp:438-476): a leaf for one light, else a node
// split at the median centre (ties by index) along the axis of widest
// centre spread; nodes numbered in preorder.
uint32_t BuildLightNode(LightBounds* first, LightBounds* last, std::vector<LightNode>& nodes) {
  if (last - first == 1) return kLightLeaf | first->index;
  const uint32_t node = static_cast<uint32_t>(nodes.size());
  nodes.emplace_back();
  double low[3], high[3];
  for (int a = 0; a < 3; ++a) low[a] = high[a] = first->centre[a];
  for (const LightBounds* it = first; it != last; ++it)
    for (int a = 0; a < 3; ++a) {
      low[a] = std::min(low[a], it->centre[a]);
      high[a] = std::max(high[a], it->centre[a]);
    }
  int axis = 0;
  for (int c = 1; c < 3; ++c)
    if (high[c] - low[c] > high[axis] - low[axis]) axis = c;
  LightBounds* middle = first + (last - first) / 2;
  std::nth_element(first, middle, last, [axis](const LightBounds& a, const LightBounds& b) {
    return a.centre[axis] != b.centre[axis] ? a.centre[axis] < b.centre[axis] : a.index < b.index;
  });
  const uint32_t left = BuildLightNode(first, middle, nodes);
  const uint32_t right = BuildLightNode(middle, last, nodes);
  LightNode& stored = nodes[node];
  StoreBounds(stored.low0, stored.high0, first, middle, left);
  StoreBounds(stored.low1, stored.high1, middle, last, right);
  return node;
}

// BuildLightHierarchy (gpu_scene.cpp:478-499).
void BuildLightHierarchy(oracle_scene& s) {
  s.light_nodes.clear();
  s.distant.clear();
  std::vector<LightBounds> bounded;
  for (size_t i = 0; i < s.analytic.size(); ++i) {
    const uint32_t shape = s.analytic[i].shape;
    if (shape == kDistantLight)
      s.distant.push_back(static_cast<uint32_t>(i));
    else if (shape != kParallelLight)
      bounded.push_back(BoundLight(s.analytic[i], static_cast<uint32_t>(i)));
  }
  if (bounded.size() == 1) {
    LightNode root;
    StoreBounds(root.low0, root.high0, bounded.data(), bounded.data() + 1, kLightLeaf | bounded[0].index);
    StoreBounds(root.low1, root.high1, nullptr, nullptr, kNoLightChild);
    s.light_nodes.push_back(root);
  } else if (bounded.size() > 1) {
    BuildLightNode(bounded.data(), bounded.data() + bounded.size(), s.light_nodes);
  }
}

// BuildLightTable (gpu_scene.cpp:515-610): emissive triangles, analytic
// lights, then the environment image.
void BuildLightTable(oracle_scene& s) {
  s.light_offsets.assign(s.instances.size(), kNoLights);
  s.lights.clear();
  std::vector<double> weights;
  for (size_t index = 0; index < s.instances.size(); ++index) {
    const Instance& inst = s.instances[index];
    const Geometry& g = s.geometries[inst.geometry];
    const double emission = EmissionEstimate(s, s.materials[inst.material]);
    const uint32_t tris = static_cast<uint32_t>(g.triangles.size() / 3);
    if (emission <= 0.0 || tris == 0) continue;
    s.light_offsets[index] = static_cast<uint32_t>(s.lights.size());
    for (uint32_t t = 0; t < tris; ++t) {
      weights.push_back(emission * WorldTriangleArea(g, t, inst.m));
      s.lights.push_back({0.0f, 1.0f, 0, static_cast<uint32_t>(index)});
    }
  }
  const double environment_mean = s.env.mean;
  bool distant = environment_mean > 0.0;
  for (const lotus_light& l : s.light_inputs) distant = distant || l.shape == LOTUS_LIGHT_DISTANT;
  const double scene_radius = distant ? SceneRadius(s) : 0.0;
  s.analytic.clear();
  std::vector<uint32_t> analytic_entries;
  for (const lotus_light& l : s.light_inputs) {
    double weight = 0.0;
    AnalyticLight record;
    if (!MakeAnalyticLight(l, scene_radius, weight, record)) continue;
    if (weight > 0.0) {
      analytic_entries.push_back(static_cast<uint32_t>(s.lights.size()));
      weights.push_back(weight);
      s.lights.push_back({0.0f, 1.0f, 0, kAnalyticLight | static_cast<uint32_t>(s.analytic.size())});
    }
    s.analytic.push_back(record);
  }
  BuildLightHierarchy(s);
  double environment_weight = 0.0;
  if (environment_mean > 0.0) {
    constexpr double kPiD = 3.14159265358979323846;
    environment_weight = kPiD * kPiD * scene_radius * scene_radius * environment_mean;
    if (!std::isfinite(environment_weight))
      environment_weight = std::numeric_limits<double>::max();
  }
  if (environment_weight > 0.0) {
    weights.push_back(environment_weight);
    s.lights.push_back({0.0f, 1.0f, 0, kEnvironmentLight});
  }
  double total = 0.0;
  for (double w : weights) total += w;
  s.environment_selection = 0.0f;
  if (!(total > 0.0) || !std::isfinite(total)) {
    s.light_offsets.assign(s.instances.size(), kNoLights);
    s.lights.clear();
    return;
  }
  const size_t count = s.lights.size();
  std::vector<double> scaled(count);
  std::vector<uint32_t> small, large;
  for (size_t i = 0; i < count; ++i) {
    s.lights[i].pdf = static_cast<float>(weights[i] / total);
    scaled[i] = weights[i] / total * static_cast<double>(count);
    (scaled[i] < 1.0 ? small : large).push_back(static_cast<uint32_t>(i));
  }
  while (!small.empty() && !large.empty()) {
    const uint32_t less = small.back();
    small.pop_back();
    const uint32_t more = large.back();
    s.lights[less].threshold = static_cast<float>(scaled[less]);
    s.lights[less].alias = more;
    scaled[more] -= 1.0 - scaled[less];
    if (scaled[more] < 1.0) {
      large.pop_back();
      small.push_back(more);
    }
  }
  for (uint32_t i : small) { s.lights[i].threshold = 1.0f; s.lights[i].alias = i; }
  for (uint32_t i : large) { s.lights[i].threshold = 1.0f; s.lights[i].alias = i; }
  for (uint32_t entry : analytic_entries)
    s.analytic[s.lights[entry].instance & ~kAnalyticLight].radiance[3] = s.lights[entry].pdf;
  if (environment_weight > 0.0) s.environment_selection = s.lights.back().pdf;
}

// ---------------------------------------------------------------------------
// Traversal

struct Ray {
  F3 origin;
  float tmin;
  F3 direction;
  float tmax;
};

struct Hit {
  uint32_t instance = 0;
  uint32_t primitive = 0;
  float b1 = 0.0f, b2 = 0.0f;
  float t = 0.0f;
};

struct Counters {
  uint64_t nodes = 0;
  uint64_t triangles = 0;
};

// The watertight ray/triangle test (Woop, Benthin and Wald, "Watertight
// Ray/Triangle Intersection", JCGT 2(1), 2013), with its double-precision
// fallback on an edge.
struct WatertightRay {
  F3 org;
  int kx, ky, kz;
  float sx, sy, sz;
};

inline WatertightRay PrepareRay(F3 org, F3 dir) {
  WatertightRay w;
  w.org = org;
  const float ax = std::fabs(dir.x), ay = std::fabs(dir.y), az = std::fabs(dir.z);
  w.kz = ax > ay ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
  w.kx = w.kz == 2 ? 0 : w.kz + 1;
  w.ky = w.kx == 2 ? 0 : w.kx + 1;
  if (Component(dir, w.kz) < 0.0f) std::swap(w.kx, w.ky);
  const float dz = Component(dir, w.kz);
  w.sx = Component(dir, w.kx) / dz;
  w.sy = Component(dir, w.ky) / dz;
  w.sz = 1.0f / dz;
  return w;
}

inline bool IntersectTriangle(const WatertightRay& r, F3 v0, F3 v1, F3 v2,
    float& t, float& b1, float& b2) {
  const F3 A = v0 - r.org, B = v1 - r.org, C = v2 - r.org;
  const float Akz = Component(A, r.kz), Bkz = Component(B, r.kz), Ckz = Component(C, r.kz);
  const float Ax = Component(A, r.kx) - r.sx * Akz;
  const float Ay = Component(A, r.ky) - r.sy * Akz;
  const float Bx = Component(B, r.kx) - r.sx * Bkz;
  const float By = Component(B, r.ky) - r.sy * Bkz;
  const float Cx = Component(C, r.kx) - r.sx * Ckz;
  const float Cy = Component(C, r.ky) - r.sy * Ckz;
  float U = Cx * By - Cy * Bx;
  float Vv = Ax * Cy - Ay * Cx;
  float W = Bx * Ay - By * Ax;
  if (U == 0.0f || Vv == 0.0f || W == 0.0f) {
    U = static_cast<float>(double(Cx) * double(By) - double(Cy) * double(Bx));
    Vv = static_cast<float>(double(Ax) * double(Cy) - double(Ay) * double(Cx));
    W = static_cast<float>(double(Bx) * double(Ay) - double(By) * double(Ax));
  }
  if ((U < 0.0f || Vv < 0.0f || W < 0.0f) && (U > 0.0f || Vv > 0.0f || W > 0.0f)) return false;
  const float det = U + Vv + W;
  if (det == 0.0f) return false;
  const float Az = r.sz * Akz, Bz = r.sz * Bkz, Cz = r.sz * Ckz;
  const float T = U * Az + Vv * Bz + W * Cz;
  const float rcp = 1.0f / det;
  t = T * rcp;
  b1 = Vv * rcp;
  b2 = W * rcp;
  return true;
}

// Whether the segment [tmin, tmax] meets the box. The far distance gets a
// relative margin of 2^-18, so that a box is never culled where the
// triangle test (whose distances carry their own rounding) could still
// accept a hit: only triangle tests decide hits, whatever the BVH.
inline bool OverlapsBox(const Box& b, F3 org, F3 inv, float tmin, float tmax) {
  const float o[3] = {org.x, org.y, org.z};
  const float d[3] = {inv.x, inv.y, inv.z};
  float t0 = tmin, t1 = tmax;
  for (int a = 0; a < 3; ++a) {
    float tn = (b.lo[a] - o[a]) * d[a];
    float tf = (b.hi[a] - o[a]) * d[a];
    if (tn > tf) std::swap(tn, tf);
    t0 = tn > t0 ? tn : t0;
    t1 = tf < t1 ? tf : t1;
  }
  return t0 <= t1 + std::fabs(t1) * 3.8146973e-6f;
}

inline F3 Inverse(F3 d) {
  auto inv = [](float x) {
    return 1.0f / (std::fabs(x) > 1e-30f ? x : (x < 0.0f ? -1e-30f : 1e-30f));
  };
  return V(inv(d.x), inv(d.y), inv(d.z));
}

// A lookup's texel at integer (x, y) after each axis's wrap: transparent
// black outside the image (LOTUS_WRAP_BLACK), the edge texel, the
// coordinate modulo the size, or mirrored every size texels (the Vulkan
// sampler address modes, vulkan_backend.cpp:3038-3053).
int32_t WrapTexel(int32_t i, int32_t n, uint32_t mode) {
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

struct Rgba {
  float v[4];
};

Rgba TexelAt(const Texture& t, int32_t x, int32_t y, uint32_t wrap_s, uint32_t wrap_t) {
  const int32_t xi = WrapTexel(x, static_cast<int32_t>(t.width), wrap_s);
  const int32_t yi = WrapTexel(y, static_cast<int32_t>(t.height), wrap_t);
  if (xi < 0 || yi < 0) return Rgba{{0.0f, 0.0f, 0.0f, 0.0f}};
  const float* p = &t.rgba[4 * (size_t{static_cast<uint32_t>(yi)} * t.width + static_cast<uint32_t>(xi))];
  return Rgba{{p[0], p[1], p[2], p[3]}};
}

// Lookup (scene.slang:315-328): the bilinear texel at (s, t), texel
// centres at (i + 1/2) / size and rows from the image's top, times scale
// plus bias; the unscaled fallback when the input names no image.
Rgba Lookup(const oracle_scene& s, const lotus_texture_input& in, float st_s, float st_t) {
  if (in.texture == LOTUS_NO_TEXTURE) return Rgba{{in.fallback[0], in.fallback[1], in.fallback[2], in.fallback[3]}};
  const float* m = in.st_transform;
  const float u = m[0] * st_s + m[1] * st_t + m[2];
  const float v = 1.0f - (m[3] * st_s + m[4] * st_t + m[5]);
  const Texture& t = s.textures[in.texture - 1];
  const float x = std::fmin(std::fmax(u * static_cast<float>(t.width) - 0.5f, -16777216.0f), 16777216.0f);
  const float y = std::fmin(std::fmax(v * static_cast<float>(t.height) - 0.5f, -16777216.0f), 16777216.0f);
  const float fx = std::floor(x), fy = std::floor(y);
  const float ax = x - fx, ay = y - fy;
  const int32_t ix = static_cast<int32_t>(fx), iy = static_cast<int32_t>(fy);
  const Rgba t00 = TexelAt(t, ix, iy, in.wrap_s, in.wrap_t);
  const Rgba t10 = TexelAt(t, ix + 1, iy, in.wrap_s, in.wrap_t);
  const Rgba t01 = TexelAt(t, ix, iy + 1, in.wrap_s, in.wrap_t);
  const Rgba t11 = TexelAt(t, ix + 1, iy + 1, in.wrap_s, in.wrap_t);
  const float bx = 1.0f - ax, by = 1.0f - ay;
  Rgba r;
  for (int c = 0; c < 4; ++c) {
    const float top = t00.v[c] * bx + t10.v[c] * ax;
    const float bottom = t01.v[c] * bx + t11.v[c] * ax;
    const float f = top * by + bottom * ay;
    r.v[c] = f * in.scale[c] + in.bias[c];
  }
  return r;
}

inline float Saturate(float x) { return std::fmin(std::fmax(x, 0.0f), 1.0f); }

// HitTexcoords (scene.slang:362-374): the instance's set interpolated with
// the barycentrics, or the material's fallback.
void HitTexcoords(const oracle_scene& s, uint32_t instance, uint32_t primitive, float b1, float b2, float& st_s,
    float& st_t) {
  const Instance& inst = s.instances[instance];
  const Geometry& g = s.geometries[inst.geometry];
  const lotus_material& m = s.materials[inst.material];
  if (inst.texcoord_set == LOTUS_NO_TEXCOORDS || inst.texcoord_set > g.texcoord_sets) {
    st_s = m.texcoord_fallback[0];
    st_t = m.texcoord_fallback[1];
    return;
  }
  const size_t tris = g.triangles.size() / 3;
  const float* c = &g.texcoords[6 * ((inst.texcoord_set - 1) * tris + primitive)];
  st_s = c[0] + b1 * (c[2] - c[0]) + b2 * (c[4] - c[0]);
  st_t = c[1] + b1 * (c[3] - c[1]) + b2 * (c[5] - c[1]);
}

// Coverage (scene.slang:393-406): the material's opacity, or its lookup's
// channel at the hit (saturated, 0 where it overflows); binary under a
// threshold.
inline float Coverage(const oracle_scene& s, uint32_t instance, uint32_t primitive, float b1, float b2) {
  const lotus_material& m = s.materials[s.instances[instance].material];
  float opacity = m.opacity;
  const uint32_t lookup = m.lookups[LOTUS_SLOT_OPACITY];
  if (lookup != LOTUS_NO_LOOKUP) {
    float st_s, st_t;
    HitTexcoords(s, instance, primitive, b1, b2, st_s, st_t);
    const lotus_texture_input& in = s.inputs[lookup - 1];
    opacity = Lookup(s, in, st_s, st_t).v[in.channel];
    opacity = std::isfinite(opacity) ? Saturate(opacity) : 0.0f;
  }
  const float threshold = m.opacity_threshold;
  if (threshold > 0.0f) return opacity >= threshold ? 1.0f : 0.0f;
  return opacity;
}

// AcceptSurface (scene.slang:408-413).
inline bool AcceptSurface(const oracle_scene& s, uint32_t instance, uint32_t primitive, float b1, float b2,
    uint32_t& rng) {
  const float coverage = Coverage(s, instance, primitive, b1, b2);
  if (coverage <= 0.0f) return false;
  if (coverage >= 1.0f) return true;
  return NextRandom(rng) < coverage;
}

inline F3 ObjectPoint(const float* inv, F3 p) {
  return V(inv[0] * p.x + inv[1] * p.y + inv[2] * p.z + inv[3],
           inv[4] * p.x + inv[5] * p.y + inv[6] * p.z + inv[7],
           inv[8] * p.x + inv[9] * p.y + inv[10] * p.z + inv[11]);
}
inline F3 ObjectVector(const float* inv, F3 d) {
  return V(inv[0] * d.x + inv[1] * d.y + inv[2] * d.z,
           inv[4] * d.x + inv[5] * d.y + inv[6] * d.z,
           inv[8] * d.x + inv[9] * d.y + inv[10] * d.z);
}

// Visits every triangle the ray's segment may meet, in BVH order, calling
// `candidate(instance, primitive, t, b1, b2)` for each intersection with t
// in [tmin, limit()]. `candidate` returns false to end the traversal.
template <typename Candidate, typename Limit>
void Traverse(const oracle_scene& s, const Ray& ray, Candidate&& candidate,
    Limit&& limit, Counters* counters) {
  if (s.tlas.nodes.empty() || s.instances.empty()) return;
  const F3 inv_world = Inverse(ray.direction);
  uint32_t stack[128];
  int top = 0;
  stack[top++] = 0;
  while (top > 0) {
    const Bvh::Node& node = s.tlas.nodes[stack[--top]];
    if (counters) ++counters->nodes;
    if (!OverlapsBox(node.box, ray.origin, inv_world, ray.tmin, limit())) continue;
    if (node.count == 0) {
      stack[top++] = node.left + 1;
      stack[top++] = node.left;
      continue;
    }
    for (uint32_t k = 0; k < node.count; ++k) {
      const uint32_t ii = s.tlas.order[node.first + k];
      const Instance& inst = s.instances[ii];
      const Geometry& g = s.geometries[inst.geometry];
      if (g.bvh.nodes.empty() || g.triangles.empty()) continue;
      const F3 o = ObjectPoint(inst.inv, ray.origin);
      const F3 d = ObjectVector(inst.inv, ray.direction);
      const WatertightRay w = PrepareRay(o, d);
      const F3 inv = Inverse(d);
      uint32_t bstack[128];
      int btop = 0;
      bstack[btop++] = 0;
      while (btop > 0) {
        const Bvh::Node& bn = g.bvh.nodes[bstack[--btop]];
        if (counters) ++counters->nodes;
        if (!OverlapsBox(bn.box, o, inv, ray.tmin, limit())) continue;
        if (bn.count == 0) {
          bstack[btop++] = bn.left + 1;
          bstack[btop++] = bn.left;
          continue;
        }
        for (uint32_t j = 0; j < bn.count; ++j) {
          const uint32_t p = g.bvh.order[bn.first + j];
          if (counters) ++counters->triangles;
          float t, b1, b2;
          if (!IntersectTriangle(w, g.positions[g.triangles[3 * p]],
                  g.positions[g.triangles[3 * p + 1]],
                  g.positions[g.triangles[3 * p + 2]], t, b1, b2))
            continue;
          if (!(t >= ray.tmin) || !(t <= limit())) continue;
          if (!candidate(ii, p, t, b1, b2)) return;
        }
      }
    }
  }
}

// Trace (scene.slang:424-439): the closest accepted hit.
bool Trace(const oracle_scene& s, const Ray& ray, uint32_t& rng, Hit& hit,
    Counters* counters = nullptr) {
  bool found = false;
  float best = ray.tmax;
  Hit h;
  Traverse(s, ray,
      [&](uint32_t ii, uint32_t p, float t, float b1, float b2) {
        if (found && (t > best || (t == best &&
                (ii > h.instance || (ii == h.instance && p >= h.primitive)))))
          return true;
        if (!AcceptSurface(s, ii, p, b1, b2, rng)) return true;
        found = true;
        best = t;
        h.instance = ii;
        h.primitive = p;
        h.b1 = b1;
        h.b2 = b2;
        h.t = t;
        return true;
      },
      [&]() { return best; }, counters);
  hit = found ? h : Hit{};
  return found;
}

// ShadowTransmittance (scene.slang:445-460).
float ShadowTransmittance(const oracle_scene& s, const Ray& ray) {
  float transmittance = 1.0f;
  bool blocked = false;
  Traverse(s, ray,
      [&](uint32_t ii, uint32_t p, float, float b1, float b2) {
        const float coverage = Coverage(s, ii, p, b1, b2);
        if (coverage >= 1.0f) {
          blocked = true;
          return false;
        }
        if (coverage > 0.0f) transmittance *= 1.0f - coverage;
        return true;
      },
      [&]() { return ray.tmax; }, nullptr);
  return blocked ? 0.0f : transmittance;
}

// ---------------------------------------------------------------------------
// Hits, lights and the environment

struct SurfaceHit {
  F3 position;
  F3 normal;
  F3 shading_normal;
  float area;
  F3 base_color;
  float roughness;
  float metallic;
  PreviewClosure bsdf;
  F3 emission;
  // A glTF PBR surface's closure, built from its terms (MakeBsdfClosure,
  // bsdf.slang:42-50); `bsdf` then holds the placeholder preview closure.
  bool gltf = false;
  ComposedClosure composed;
  GltfPbrTerms gltf_terms;
};

// BsdfEvaluate, BsdfPdf and BsdfSample (bsdf.slang:52-90).
F3 BsdfEvaluate(const SurfaceHit& sh, F3 wo, F3 wi) {
  return sh.gltf ? ComposedEvaluate(sh.composed, wo, wi) : PreviewEvaluate(sh.bsdf, wo, wi);
}

float BsdfPdf(const SurfaceHit& sh, F3 wo, F3 wi) {
  return sh.gltf ? ComposedPdf(sh.composed, wo, wi) : PreviewPdf(sh.bsdf, wo, wi);
}

bool BsdfSample(const SurfaceHit& sh, F3 wo, F3 u, BsdfSampleResult& s) {
  return sh.gltf ? ComposedSample(sh.composed, wo, u, s) : PreviewSample(sh.bsdf, wo, u, s);
}

// OffsetRayOrigin (scene.slang:1454-1469).
F3 OffsetRayOrigin(F3 position, F3 normal) {
  constexpr float kOrigin = 1.0f / 32.0f;
  constexpr float kFloatScale = 1.0f / 65536.0f;
  constexpr float kIntScale = 256.0f;
  float p[3] = {position.x, position.y, position.z};
  const float n[3] = {normal.x, normal.y, normal.z};
  float r[3];
  for (int a = 0; a < 3; ++a) {
    const int offset = static_cast<int>(kIntScale * n[a]);
    const float moved = AsFloat(static_cast<uint32_t>(
        static_cast<int32_t>(AsUint(p[a])) + (p[a] < 0.0f ? -offset : offset)));
    r[a] = std::fabs(p[a]) < kOrigin ? p[a] + kFloatScale * n[a] : moved;
  }
  return V(r[0], r[1], r[2]);
}

// ShadingNormal (scene.slang:467-488).
F3 ShadingNormal(const F3* n, float b1, float b2, const float* m, F3 geometric, F3 direction) {
  const F3 object = n[0] + b1 * (n[1] - n[0]) + b2 * (n[2] - n[0]);
  const F3 c0 = V(m[0], m[1], m[2]);
  const F3 c1 = V(m[4], m[5], m[6]);
  const F3 c2 = V(m[8], m[9], m[10]);
  const F3 world = cross(c1, c2) * object.x + cross(c2, c0) * object.y + cross(c0, c1) * object.z;
  const float length2 = dot(world, world);
  if (!(length2 > 0.0f) || std::isinf(length2)) return geometric;
  F3 shading = world * rsqrt(length2);
  if (dot(shading, geometric) < 0.0f) shading = -shading;
  return dot(shading, direction) < 0.0f ? shading : geometric;
}

inline float TriangleArea(F3 p0, F3 p1, F3 p2) { return 0.5f * length(cross(p1 - p0, p2 - p0)); }

// PreviewEmission (scene.slang:570-577): the constant, or the lookup's RGB
// at (st_s, st_t) with negative parts cut.
F3 PreviewEmission(const oracle_scene& s, const lotus_material& m, float st_s, float st_t) {
  const uint32_t lookup = m.lookups[LOTUS_SLOT_EMISSION];
  if (lookup == LOTUS_NO_LOOKUP) return V(m.emission[0], m.emission[1], m.emission[2]);
  const Rgba v = Lookup(s, s.inputs[lookup - 1], st_s, st_t);
  return V(std::fmax(v.v[0], 0.0f), std::fmax(v.v[1], 0.0f), std::fmax(v.v[2], 0.0f));
}

// GltfEmission (scene.slang:579-588): emissive or its lookup, times the
// strength.
F3 GltfEmission(const oracle_scene& s, const lotus_material& m, float st_s, float st_t) {
  const float strength = m.emissive_strength;
  const uint32_t lookup = m.lookups[LOTUS_GLTF_SLOT_EMISSIVE];
  if (lookup == LOTUS_NO_LOOKUP) return V(m.emission[0], m.emission[1], m.emission[2]) * strength;
  const Rgba v = Lookup(s, s.inputs[lookup - 1], st_s, st_t);
  return V(std::fmax(v.v[0], 0.0f), std::fmax(v.v[1], 0.0f), std::fmax(v.v[2], 0.0f)) * strength;
}

// Emission (scene.slang:590-600).
F3 Emission(const oracle_scene& s, const lotus_material& m, float st_s, float st_t) {
  return m.model == LOTUS_MODEL_GLTF_PBR ? GltfEmission(s, m, st_s, st_t) : PreviewEmission(s, m, st_s, st_t);
}

inline bool Textured(const lotus_material& m) {
  for (uint32_t k = 0; k < LOTUS_TEXTURE_SLOTS; ++k)
    if (m.lookups[k] != LOTUS_NO_LOOKUP) return true;
  return !(m.normal[0] == 0.0f && m.normal[1] == 0.0f && (m.normal[2] == 0.0f || m.normal[2] == 1.0f));
}

// TangentFrame (scene.slang:490-538): the texture coordinates'
// differentials in world space, orthonormalized about the interpolated
// shading normal, keeping mirrored coordinates' handedness; the
// normal-only frame without usable coordinates. A normal-map lookup
// transforms the differentials as its coordinates.
ShadingFrame TangentFrame(const oracle_scene& s, uint32_t instance, const lotus_texture_input* input,
    uint32_t primitive, F3 edge1, F3 edge2, F3 normal) {
  ShadingFrame basis = MakeShadingFrame(normal);
  const Instance& inst = s.instances[instance];
  const Geometry& g = s.geometries[inst.geometry];
  if (inst.texcoord_set == LOTUS_NO_TEXCOORDS || inst.texcoord_set > g.texcoord_sets) return basis;
  const size_t tris = g.triangles.size() / 3;
  const float* c = &g.texcoords[6 * ((inst.texcoord_set - 1) * tris + primitive)];
  float u1 = c[2] - c[0], v1 = c[3] - c[1], u2 = c[4] - c[0], v2 = c[5] - c[1];
  if (input) {
    const float* m = input->st_transform;
    const float a1 = m[0] * u1 + m[1] * v1, b1 = m[3] * u1 + m[4] * v1;
    const float a2 = m[0] * u2 + m[1] * v2, b2 = m[3] * u2 + m[4] * v2;
    u1 = a1;
    v1 = b1;
    u2 = a2;
    v2 = b2;
  }
  const float uv_scale = std::fmax(std::fmax(std::fabs(u1), std::fabs(v1)), std::fmax(std::fabs(u2), std::fabs(v2)));
  const float edge_scale = std::fmax(std::fmax(std::fmax(std::fabs(edge1.x), std::fabs(edge1.y)), std::fabs(edge1.z)),
      std::fmax(std::fmax(std::fabs(edge2.x), std::fabs(edge2.y)), std::fabs(edge2.z)));
  if (!(uv_scale > 0.0f) || std::isinf(uv_scale) || !(edge_scale > 0.0f) || std::isinf(edge_scale)) return basis;
  u1 = u1 / uv_scale;
  v1 = v1 / uv_scale;
  u2 = u2 / uv_scale;
  v2 = v2 / uv_scale;
  edge1 = V(edge1.x / edge_scale, edge1.y / edge_scale, edge1.z / edge_scale);
  edge2 = V(edge2.x / edge_scale, edge2.y / edge_scale, edge2.z / edge_scale);
  const float determinant = u1 * v2 - v1 * u2;
  if (!(std::fabs(determinant) > 1e-8f)) return basis;
  const float orientation = determinant < 0.0f ? -1.0f : 1.0f;
  F3 tangent = orientation * (edge1 * v2 - edge2 * v1);
  const F3 bitangent = orientation * (edge2 * u1 - edge1 * u2);
  tangent = tangent - normal * dot(normal, tangent);
  const float length2 = dot(tangent, tangent);
  if (!(length2 > 1e-16f) || std::isinf(length2)) return basis;
  basis.tangent = tangent * rsqrt(length2);
  basis.bitangent = cross(normal, basis.tangent);
  if (dot(basis.bitangent, bitangent) < 0.0f) basis.bitangent = -basis.bitangent;
  return basis;
}

// MappedNormal (scene.slang:541-556).
F3 MappedNormal(F3 tangent_normal, const ShadingFrame& basis, F3 geometric, F3 direction) {
  const float magnitude =
      std::fmax(std::fmax(std::fabs(tangent_normal.x), std::fabs(tangent_normal.y)), std::fabs(tangent_normal.z));
  if (!(magnitude > 0.0f) || !std::isfinite(tangent_normal.x) || !std::isfinite(tangent_normal.y) ||
      !std::isfinite(tangent_normal.z))
    return basis.normal;
  F3 shading = normalize(basis.ToWorld(
      V(tangent_normal.x / magnitude, tangent_normal.y / magnitude, tangent_normal.z / magnitude)));
  if (dot(shading, geometric) < 0.0f) shading = -shading;
  return dot(shading, direction) < 0.0f ? shading : basis.normal;
}

// ReconstructHit + EvaluatePreview (scene.slang:1408-1449, 1184-1260): a
// texture lookup replaces its input's constant, clamped into its range.
// GltfScalar (scene.slang:1262-1274): a scalar input's lookup channel,
// clamped to [0, 1], or its constant.
float GltfScalar(const oracle_scene& s, const lotus_material& m, uint32_t slot, float st_s, float st_t,
    float constant) {
  const uint32_t k = m.lookups[slot];
  if (k == LOTUS_NO_LOOKUP) return constant;
  const lotus_texture_input& in = s.inputs[k - 1];
  return saturate(Lookup(s, in, st_s, st_t).v[in.channel]);
}

inline F3 ClampNormal(const Rgba& v) {
  return V(std::fmin(std::fmax(v.v[0], -1.0f), 1.0f), std::fmin(std::fmax(v.v[1], -1.0f), 1.0f),
      std::fmin(std::fmax(v.v[2], -1.0f), 1.0f));
}

// EvaluateGltfPbr (scene.slang:1276-1406).
void EvaluateGltfPbr(const oracle_scene& s, const Hit& hit, const lotus_material& mat, F3 edge1, F3 edge2,
    F3 direction, SurfaceHit& sh) {
  sh.base_color = V(mat.base_color[0], mat.base_color[1], mat.base_color[2]);
  sh.roughness = mat.roughness;
  sh.metallic = mat.metallic;
  F3 emission = V(mat.emission[0], mat.emission[1], mat.emission[2]) * mat.emissive_strength;
  const bool zero = mat.normal[0] == 0.0f && mat.normal[1] == 0.0f && mat.normal[2] == 0.0f;
  F3 tangent_normal = zero ? V(0.0f, 0.0f, 1.0f) : V(mat.normal[0], mat.normal[1], mat.normal[2]);
  // The dielectric's reflectance at normal incidence, which the host
  // computes in double (gpu_scene.cpp:2059-2063).
  const double root = (1.0 - double{mat.ior}) / (1.0 + double{mat.ior});
  const float dielectric_f0 = static_cast<float>(root * root);
  float specular = mat.specular;
  float transmission = mat.transmission;
  F3 specular_color = V(mat.specular_color[0], mat.specular_color[1], mat.specular_color[2]);
  float clearcoat = mat.clearcoat;
  F3 sheen_color = V(mat.sheen_color[0], mat.sheen_color[1], mat.sheen_color[2]);
  float sheen_roughness = mat.sheen_roughness;
  float clearcoat_roughness = mat.clearcoat_roughness;
  const F3 mesh_normal = sh.shading_normal;
  F3 coat_tangent_normal = V(0.0f, 0.0f, 1.0f);
  if (Textured(mat)) {
    float st_s, st_t;
    HitTexcoords(s, hit.instance, hit.primitive, hit.b1, hit.b2, st_s, st_t);
    uint32_t k = mat.lookups[LOTUS_GLTF_SLOT_BASE_COLOR];
    if (k != LOTUS_NO_LOOKUP) {
      const Rgba v = Lookup(s, s.inputs[k - 1], st_s, st_t);
      sh.base_color = V(saturate(v.v[0]), saturate(v.v[1]), saturate(v.v[2]));
    }
    sh.roughness = GltfScalar(s, mat, LOTUS_GLTF_SLOT_ROUGHNESS, st_s, st_t, sh.roughness);
    sh.metallic = GltfScalar(s, mat, LOTUS_GLTF_SLOT_METALLIC, st_s, st_t, sh.metallic);
    emission = GltfEmission(s, mat, st_s, st_t);
    k = mat.lookups[LOTUS_SLOT_NORMAL];
    if (k != LOTUS_NO_LOOKUP) tangent_normal = ClampNormal(Lookup(s, s.inputs[k - 1], st_s, st_t));
    specular = GltfScalar(s, mat, LOTUS_GLTF_SLOT_SPECULAR, st_s, st_t, specular);
    transmission = GltfScalar(s, mat, LOTUS_GLTF_SLOT_TRANSMISSION, st_s, st_t, transmission);
    clearcoat = GltfScalar(s, mat, LOTUS_GLTF_SLOT_CLEARCOAT, st_s, st_t, clearcoat);
    clearcoat_roughness = GltfScalar(s, mat, LOTUS_GLTF_SLOT_CLEARCOAT_ROUGHNESS, st_s, st_t, clearcoat_roughness);
    sheen_roughness = GltfScalar(s, mat, LOTUS_GLTF_SLOT_SHEEN_ROUGHNESS, st_s, st_t, sheen_roughness);
    k = mat.lookups[LOTUS_GLTF_SLOT_SPECULAR_COLOR];
    if (k != LOTUS_NO_LOOKUP) {
      const Rgba v = Lookup(s, s.inputs[k - 1], st_s, st_t);
      specular_color = V(std::fmax(v.v[0], 0.0f), std::fmax(v.v[1], 0.0f), std::fmax(v.v[2], 0.0f));
    }
    k = mat.lookups[LOTUS_GLTF_SLOT_SHEEN_COLOR];
    if (k != LOTUS_NO_LOOKUP) {
      const Rgba v = Lookup(s, s.inputs[k - 1], st_s, st_t);
      sheen_color = V(saturate(v.v[0]), saturate(v.v[1]), saturate(v.v[2]));
    }
    k = mat.lookups[LOTUS_GLTF_SLOT_CLEARCOAT_NORMAL];
    if (k != LOTUS_NO_LOOKUP) coat_tangent_normal = ClampNormal(Lookup(s, s.inputs[k - 1], st_s, st_t));
  }
  if (tangent_normal.x != 0.0f || tangent_normal.y != 0.0f || tangent_normal.z != 1.0f) {
    const uint32_t k = mat.lookups[LOTUS_SLOT_NORMAL];
    sh.shading_normal = MappedNormal(tangent_normal,
        TangentFrame(s, hit.instance, k != LOTUS_NO_LOOKUP ? &s.inputs[k - 1] : nullptr, hit.primitive, edge1,
            edge2, sh.shading_normal),
        sh.normal, direction);
  }
  const float cos_o = dot(sh.shading_normal, -direction);
  F3 wo = V(std::sqrt(std::fmax(1.0f - cos_o * cos_o, 0.0f)), 0.0f, cos_o);
  GltfPbrInputs inputs = MakeGltfPbrInputs(sh.base_color, sh.roughness, sh.metallic);
  inputs.dielectric_f0 = dielectric_f0;
  inputs.specular = specular;
  inputs.specular_color = specular_color;
  inputs.transmission = transmission;
  inputs.clearcoat = clearcoat;
  inputs.clearcoat_roughness = clearcoat_roughness;
  inputs.sheen_color = sheen_color;
  inputs.sheen_roughness = sheen_roughness;
  if (clearcoat > 0.0f) {
    F3 coat_normal = mesh_normal;
    if (coat_tangent_normal.x != 0.0f || coat_tangent_normal.y != 0.0f || coat_tangent_normal.z != 1.0f) {
      const uint32_t k = mat.lookups[LOTUS_GLTF_SLOT_CLEARCOAT_NORMAL];
      coat_normal = MappedNormal(coat_tangent_normal,
          TangentFrame(s, hit.instance, k != LOTUS_NO_LOOKUP ? &s.inputs[k - 1] : nullptr, hit.primitive,
              edge1, edge2, mesh_normal),
          sh.normal, direction);
    }
    const ShadingFrame basis = MakeShadingFrame(sh.shading_normal);
    const F3 local = basis.ToLocal(-direction);
    wo.x = local.x;
    wo.y = local.y;
    inputs.clearcoat_normal = normalize(basis.ToLocal(coat_normal));
  }
  sh.gltf_terms = MakeGltfPbrTerms(inputs, wo);
  sh.composed = MakeGltfPbrClosure(sh.gltf_terms, wo);
  sh.gltf = true;
  sh.bsdf = MakePreviewClosure(V(0.0f), 1.0f, 0.0f, 1.5f, false, V(0.0f), 0.0f, V(1.0f), false, true);
  sh.emission = emission;
}

// HitColor (scene.slang:376-386).
F3 HitColor(const std::vector<F3>& set, uint32_t primitive, float b1, float b2) {
  if (set.size() == 1) return set[0];
  const F3 c0 = set[3 * primitive], c1 = set[3 * primitive + 1], c2 = set[3 * primitive + 2];
  return c0 + b1 * (c1 - c0) + b2 * (c2 - c0);
}

SurfaceHit ReconstructHit(const oracle_scene& s, const Hit& hit, F3 direction) {
  const Instance& inst = s.instances[hit.instance];
  const Geometry& g = s.geometries[inst.geometry];
  const uint32_t* tri = &g.triangles[3 * hit.primitive];
  const F3 p0 = TransformPoint(inst.m, g.positions[tri[0]]);
  const F3 p1 = TransformPoint(inst.m, g.positions[tri[1]]);
  const F3 p2 = TransformPoint(inst.m, g.positions[tri[2]]);
  SurfaceHit sh;
  sh.position = p0 + hit.b1 * (p1 - p0) + hit.b2 * (p2 - p0);
  const F3 normal = normalize(cross(p1 - p0, p2 - p0));
  sh.area = TriangleArea(p0, p1, p2);
  sh.normal = dot(normal, direction) > 0.0f ? -normal : normal;
  sh.shading_normal = sh.normal;
  if (!g.normals.empty())
    sh.shading_normal = ShadingNormal(&g.normals[3 * hit.primitive], hit.b1, hit.b2,
        inst.m, sh.normal, direction);
  const lotus_material& mat = s.materials[inst.material];
  if (mat.model == LOTUS_MODEL_GLTF_PBR) {
    EvaluateGltfPbr(s, hit, mat, p1 - p0, p2 - p0, direction, sh);
    return sh;
  }
  sh.base_color = V(mat.base_color[0], mat.base_color[1], mat.base_color[2]);
  // EvaluatePreview (scene.slang:1187-1189): the instance's colour set,
  // clamped, where it reads one.
  if (inst.color_set != LOTUS_NO_COLORS && inst.color_set <= g.colors.size()) {
    const F3 c = HitColor(g.colors[inst.color_set - 1], hit.primitive, hit.b1, hit.b2);
    sh.base_color = V(saturate(c.x), saturate(c.y), saturate(c.z));
  }
  sh.roughness = mat.roughness;
  sh.metallic = mat.metallic;
  F3 emission = V(mat.emission[0], mat.emission[1], mat.emission[2]);
  F3 specular = V(mat.specular_color[0], mat.specular_color[1], mat.specular_color[2]);
  if (Textured(mat)) {
    float st_s, st_t;
    HitTexcoords(s, hit.instance, hit.primitive, hit.b1, hit.b2, st_s, st_t);
    uint32_t k = mat.lookups[LOTUS_SLOT_BASE_COLOR];
    if (k != LOTUS_NO_LOOKUP) {
      const Rgba v = Lookup(s, s.inputs[k - 1], st_s, st_t);
      sh.base_color = V(Saturate(v.v[0]), Saturate(v.v[1]), Saturate(v.v[2]));
    }
    k = mat.lookups[LOTUS_SLOT_ROUGHNESS];
    if (k != LOTUS_NO_LOOKUP)
      sh.roughness = Saturate(Lookup(s, s.inputs[k - 1], st_s, st_t).v[s.inputs[k - 1].channel]);
    k = mat.lookups[LOTUS_SLOT_METALLIC];
    if (k != LOTUS_NO_LOOKUP)
      sh.metallic = Saturate(Lookup(s, s.inputs[k - 1], st_s, st_t).v[s.inputs[k - 1].channel]);
    emission = PreviewEmission(s, mat, st_s, st_t);
    const bool zero = mat.normal[0] == 0.0f && mat.normal[1] == 0.0f && mat.normal[2] == 0.0f;
    F3 tangent_normal = zero ? V(0.0f, 0.0f, 1.0f) : V(mat.normal[0], mat.normal[1], mat.normal[2]);
    const uint32_t normal_lookup = mat.lookups[LOTUS_SLOT_NORMAL];
    if (normal_lookup != LOTUS_NO_LOOKUP) {
      const Rgba v = Lookup(s, s.inputs[normal_lookup - 1], st_s, st_t);
      tangent_normal = V(std::fmin(std::fmax(v.v[0], -1.0f), 1.0f), std::fmin(std::fmax(v.v[1], -1.0f), 1.0f),
          std::fmin(std::fmax(v.v[2], -1.0f), 1.0f));
    }
    k = mat.lookups[LOTUS_SLOT_SPECULAR_COLOR];
    if (k != LOTUS_NO_LOOKUP) {
      const Rgba v = Lookup(s, s.inputs[k - 1], st_s, st_t);
      if (std::isfinite(v.v[0]) && std::isfinite(v.v[1]) && std::isfinite(v.v[2]))
        specular = V(Saturate(v.v[0]), Saturate(v.v[1]), Saturate(v.v[2]));
    }
    if (tangent_normal.x != 0.0f || tangent_normal.y != 0.0f || tangent_normal.z != 1.0f)
      sh.shading_normal = MappedNormal(tangent_normal,
          TangentFrame(s, hit.instance, normal_lookup != LOTUS_NO_LOOKUP ? &s.inputs[normal_lookup - 1] : nullptr,
              hit.primitive, p1 - p0, p2 - p0, sh.shading_normal),
          sh.normal, direction);
  }
  bool entering = true;
  const float transmission = mat.transmission;
  if (transmission > 0.0f) {
    const F3 c0 = V(inst.m[0], inst.m[1], inst.m[2]);
    const F3 c1 = V(inst.m[4], inst.m[5], inst.m[6]);
    const F3 c2 = V(inst.m[8], inst.m[9], inst.m[10]);
    const F3 outward = dot(c0, cross(c1, c2)) < 0.0f ? -normal : normal;
    entering = dot(outward, direction) < 0.0f;
  }
  sh.bsdf = MakePreviewClosure(sh.base_color, sh.roughness, sh.metallic, mat.ior,
      (mat.flags & LOTUS_MATERIAL_SPECULAR_WORKFLOW) != 0, specular, transmission,
      V(mat.transmission_color[0], mat.transmission_color[1], mat.transmission_color[2]),
      (mat.flags & LOTUS_MATERIAL_THIN_WALLED) != 0, entering);
  sh.emission = emission;
  return sh;
}

struct LightSample {
  F3 direction;
  float distance;
  F3 radiance;
  float pdf;
  bool delta;
};

inline LightSample NoLight() { return LightSample{V(0.0f, 0.0f, 1.0f), 0.0f, V(0.0f), 0.0f, false}; }

// SampleTriangle (scene.slang:632-677).
LightSample SampleTriangle(const oracle_scene& s, uint32_t light, const LightRecord& chosen,
    float ux, float uy, F3 origin) {
  const uint32_t primitive = light - s.light_offsets[chosen.instance];
  const float root = std::sqrt(ux);
  const float b1 = root * (1.0f - uy), b2 = root * uy;
  const Instance& inst = s.instances[chosen.instance];
  const Geometry& g = s.geometries[inst.geometry];
  const uint32_t* tri = &g.triangles[3 * primitive];
  const F3 p0 = TransformPoint(inst.m, g.positions[tri[0]]);
  const F3 p1 = TransformPoint(inst.m, g.positions[tri[1]]);
  const F3 p2 = TransformPoint(inst.m, g.positions[tri[2]]);
  const lotus_material& mat = s.materials[inst.material];
  const F3 position = p0 + b1 * (p1 - p0) + b2 * (p2 - p0);
  const F3 normal = normalize(cross(p1 - p0, p2 - p0));
  const float area = TriangleArea(p0, p1, p2);
  F3 radiance;
  if (mat.lookups[LOTUS_SLOT_EMISSION] == LOTUS_NO_LOOKUP && mat.lookups[LOTUS_SLOT_OPACITY] == LOTUS_NO_LOOKUP) {
    const float strength = mat.model == LOTUS_MODEL_GLTF_PBR ? mat.emissive_strength : 1.0f;
    const F3 e = mat.model == LOTUS_MODEL_GLTF_PBR ? V(mat.emission[0], mat.emission[1], mat.emission[2]) * strength
                                                   : V(mat.emission[0], mat.emission[1], mat.emission[2]);
    radiance = e * Coverage(s, chosen.instance, primitive, b1, b2);
  } else {
    // Emission(material, HitTexcoords) * Coverage(hit) at the sampled point
    // (scene.slang:655-657).
    float st_s, st_t;
    HitTexcoords(s, chosen.instance, primitive, b1, b2, st_s, st_t);
    radiance = Emission(s, mat, st_s, st_t) * Coverage(s, chosen.instance, primitive, b1, b2);
  }
  const F3 toward = position - origin;
  const float distance2 = dot(toward, toward);
  if (!(area > 0.0f) || !(distance2 > 0.0f) || MaxComponent(radiance) <= 0.0f) return NoLight();
  LightSample ls;
  ls.direction = toward * rsqrt(distance2);
  const float cosine = std::fabs(dot(normal, ls.direction));
  if (!(cosine > 0.0f)) return NoLight();
  const F3 end = OffsetRayOrigin(position, dot(normal, ls.direction) > 0.0f ? -normal : normal);
  ls.distance = std::fmax(0.0f, dot(end - origin, ls.direction));
  ls.radiance = radiance;
  ls.pdf = chosen.pdf / area * distance2 / cosine;
  ls.delta = false;
  return ls;
}

inline float EnvFloat(const oracle_scene& s, uint64_t index) { return s.env.floats[index]; }

// FindInterval (scene.slang:775-789).
uint32_t FindInterval(const oracle_scene& s, uint64_t first, uint32_t count, float u) {
  uint32_t low = 0;
  uint32_t len = count + 1;
  while (len > 0) {
    const uint32_t half = len >> 1;
    const uint32_t middle = low + half;
    if (EnvFloat(s, first + middle) <= u) {
      low = middle + 1;
      len -= half + 1;
    } else {
      len = half;
    }
  }
  return std::min(std::max(low, 1u), count) - 1;
}

// SampleCumulative (scene.slang:794-800).
float SampleCumulative(const oracle_scene& s, uint64_t first, uint32_t count, float u, uint32_t& cell) {
  cell = FindInterval(s, first, count, u);
  const float low = EnvFloat(s, first + cell);
  const float width = EnvFloat(s, first + cell + 1) - low;
  const float offset = width > 0.0f ? (u - low) / width : 0.5f;
  return std::fmin((float(cell) + offset) / float(count), 0.99999994f);
}

// EnvironmentUv (scene.slang:805-809).
inline void EnvironmentUv(F3 local, float& u, float& v) {
  const float uu = 0.5f - latan2(local.x, local.z) * (0.5f / kPi);
  v = lacos(std::fmin(std::fmax(local.y, -1.0f), 1.0f)) * (1.0f / kPi);
  u = uu - std::floor(uu);
}

// EnvironmentDirection (scene.slang:811-816).
inline F3 EnvironmentDirection(float u, float v) {
  const float theta = kPi * v;
  const float phi = kPi * (1.0f - 2.0f * u);
  float sin_theta, cos_theta, sin_phi, cos_phi;
  lsincos(theta, sin_theta, cos_theta);
  lsincos(phi, sin_phi, cos_phi);
  return V(sin_theta * sin_phi, cos_theta, sin_theta * cos_phi);
}

// EnvironmentLookup (scene.slang:819-824): the bilinear texel, repeating
// across longitude and clamped at the poles, times the scale.
F3 EnvironmentLookup(const oracle_scene& s, float u, float v) {
  const Environment& e = s.env;
  const float x = u * float(e.width) - 0.5f;
  const float y = v * float(e.height) - 0.5f;
  const float fx0 = std::floor(x), fy0 = std::floor(y);
  const float ax = x - fx0, ay = y - fy0;
  const int w = static_cast<int>(e.width), h = static_cast<int>(e.height);
  int x0 = static_cast<int>(fx0) % w;
  if (x0 < 0) x0 += w;
  const int x1 = x0 + 1 == w ? 0 : x0 + 1;
  const int iy = static_cast<int>(fy0);
  const int y0 = std::min(std::max(iy, 0), h - 1);
  const int y1 = std::min(std::max(iy + 1, 0), h - 1);
  const float* t00 = &e.texels[4 * (size_t(y0) * w + x0)];
  const float* t10 = &e.texels[4 * (size_t(y0) * w + x1)];
  const float* t01 = &e.texels[4 * (size_t(y1) * w + x0)];
  const float* t11 = &e.texels[4 * (size_t(y1) * w + x1)];
  float c[3];
  for (int k = 0; k < 3; ++k) {
    const float top = t00[k] * (1.0f - ax) + t10[k] * ax;
    const float bottom = t01[k] * (1.0f - ax) + t11[k] * ax;
    c[k] = top * (1.0f - ay) + bottom * ay;
  }
  return V(std::fmax(c[0], 0.0f) * e.scale.x, std::fmax(c[1], 0.0f) * e.scale.y,
      std::fmax(c[2], 0.0f) * e.scale.z);
}

// EnvironmentDirectionPdf (scene.slang:829-840).
float EnvironmentDirectionPdf(const oracle_scene& s, float u, float v) {
  const uint32_t column = std::min(static_cast<uint32_t>(u * float(s.env.columns)), s.env.columns - 1);
  const uint32_t row = std::min(static_cast<uint32_t>(v * float(s.env.rows_count)), s.env.rows_count - 1);
  const float sin_theta = lsin(kPi * v);
  if (!(sin_theta > 0.0f)) return 0.0f;
  return EnvFloat(s, uint64_t(row) * s.env.columns + column) / (2.0f * kPi * kPi * sin_theta);
}

// SampleEnvironment (scene.slang:845-872).
LightSample SampleEnvironment(const oracle_scene& s, float selection, float ux, float uy) {
  const Environment& e = s.env;
  const uint64_t cells = uint64_t(e.columns) * e.rows_count;
  uint32_t row, column;
  const float v = SampleCumulative(s, cells, e.rows_count, ux, row);
  const float u = SampleCumulative(s, cells + e.rows_count + 1 + uint64_t(row) * (e.columns + 1),
      e.columns, uy, column);
  const float sin_theta = lsin(kPi * v);
  const float density = EnvFloat(s, uint64_t(row) * e.columns + column);
  if (!(sin_theta > 0.0f) || !(density > 0.0f)) return NoLight();
  const F3 local = EnvironmentDirection(u, v);
  LightSample ls;
  ls.direction = normalize(local.x * e.rows[0] + local.y * e.rows[1] + local.z * e.rows[2]);
  ls.distance = kFloatMax;
  ls.radiance = EnvironmentLookup(s, u, v);
  ls.pdf = selection * density / (2.0f * kPi * kPi * sin_theta);
  ls.delta = false;
  return ls;
}

// EnvironmentRadiance (scene.slang:877-890).
F3 EnvironmentRadiance(const oracle_scene& s, F3 direction, bool weigh, float pdf) {
  const Environment& e = s.env;
  const F3 local = V(dot(e.rows[0], direction), dot(e.rows[1], direction), dot(e.rows[2], direction));
  float u, v;
  EnvironmentUv(local, u, v);
  const F3 radiance = EnvironmentLookup(s, u, v);
  if (!weigh || !(s.environment_selection > 0.0f)) return radiance;
  return radiance * PowerHeuristic(pdf, s.environment_selection * EnvironmentDirectionPdf(s, u, v));
}

// SampleConcentricDisk (sampling.slang:89-104).
inline void SampleConcentricDisk(float ux, float uy, float& a, float& b) {
  const float ox = 2.0f * ux - 1.0f, oy = 2.0f * uy - 1.0f;
  if (ox == 0.0f && oy == 0.0f) {
    a = b = 0.0f;
    return;
  }
  float radius, theta;
  if (std::fabs(ox) > std::fabs(oy)) {
    radius = ox;
    theta = 0.25f * kPi * (oy / ox);
  } else {
    radius = oy;
    theta = 0.5f * kPi - 0.25f * kPi * (ox / oy);
  }
  float sn, cs;
  lsincos(theta, sn, cs);
  a = radius * cs;
  b = radius * sn;
}

// SampleUniformCone (sampling.slang:109-116).
inline F3 SampleUniformCone(float ux, float uy, float one_minus_cos_max) {
  const float one_minus_cos = ux * one_minus_cos_max;
  const float sin_theta = std::sqrt(std::fmax(0.0f, one_minus_cos * (2.0f - one_minus_cos)));
  const float phi = 2.0f * kPi * uy;
  float sn, cs;
  lsincos(phi, sn, cs);
  return V(sin_theta * cs, sin_theta * sn, 1.0f - one_minus_cos);
}

inline F3 Xyz4(const float* v) { return V(v[0], v[1], v[2]); }

// SphereConePdf (scene.slang:683-690).
inline float SphereConePdf(float sin2_max) {
  const float one_minus_cos = sin2_max < 0.00068523f ? 0.5f * sin2_max
                                                     : 1.0f - std::sqrt(std::fmax(0.0f, 1.0f - sin2_max));
  return 1.0f / (2.0f * kPi * one_minus_cos);
}

// SampleAnalytic (scene.slang:695-768).
LightSample SampleAnalytic(const AnalyticLight& light, float selection, float ux, float uy, F3 origin) {
  LightSample ls = NoLight();
  ls.radiance = Xyz4(light.radiance);
  if (light.shape == kSphereLight) {
    const F3 centre = Xyz4(light.position);
    const float radius = light.position[3];
    const F3 to_centre = centre - origin;
    const float distance2 = dot(to_centre, to_centre);
    if (!(distance2 > radius * radius)) return NoLight();
    const float sin2_max = radius * radius / distance2;
    const float sin_max = std::sqrt(sin2_max);
    const float cos_max = std::sqrt(std::fmax(0.0f, 1.0f - sin2_max));
    float cos_theta = (cos_max - 1.0f) * ux + 1.0f;
    float sin2_theta = 1.0f - cos_theta * cos_theta;
    if (sin2_max < 0.00068523f) {
      sin2_theta = sin2_max * ux;
      cos_theta = std::sqrt(1.0f - sin2_theta);
    }
    const float cos_alpha = sin2_theta / sin_max +
        cos_theta * std::sqrt(std::fmax(0.0f, 1.0f - sin2_theta / sin2_max));
    const float sin_alpha = std::sqrt(std::fmax(0.0f, 1.0f - cos_alpha * cos_alpha));
    const float phi = 2.0f * kPi * uy;
    float sn, cs;
    lsincos(phi, sn, cs);
    const ShadingFrame frame = MakeShadingFrame(normalize(to_centre));
    const F3 outward = frame.ToWorld(-V(sin_alpha * cs, sin_alpha * sn, cos_alpha));
    const F3 toward = centre + radius * outward - origin;
    ls.distance = length(toward);
    ls.direction = toward / ls.distance;
    ls.pdf = selection * SphereConePdf(sin2_max);
  } else if (light.shape == kRectLight || light.shape == kDiskLight) {
    float a, b;
    if (light.shape == kRectLight) {
      a = 2.0f * ux - 1.0f;
      b = 2.0f * uy - 1.0f;
    } else {
      SampleConcentricDisk(ux, uy, a, b);
    }
    const F3 toward = Xyz4(light.position) + a * Xyz4(light.axis_u) + b * Xyz4(light.axis_v) - origin;
    const float distance2 = dot(toward, toward);
    if (!(distance2 > 0.0f)) return NoLight();
    ls.distance = std::sqrt(distance2);
    ls.direction = toward / ls.distance;
    const float cosine = -dot(Xyz4(light.normal), ls.direction);
    if (!(cosine > 0.0f)) return NoLight();
    ls.pdf = selection * distance2 / (cosine * light.normal[3]);
  } else if (light.shape == kDistantLight) {
    const ShadingFrame frame = MakeShadingFrame(Xyz4(light.axis_u));
    ls.direction = normalize(frame.ToWorld(SampleUniformCone(ux, uy, light.axis_u[3])));
    ls.distance = kFloatMax;
    ls.pdf = selection / (2.0f * kPi * light.axis_u[3]);
  } else {
    ls.direction = Xyz4(light.axis_u);
    ls.distance = kFloatMax;
    ls.pdf = selection;
    ls.delta = true;
  }
  return ls;
}

// ParallelLight (scene.slang:986-1000).
LightSample ParallelLight(const oracle_scene& s, uint32_t index) {
  const AnalyticLight& light = s.analytic[index];
  if (light.shape != kParallelLight) return NoLight();
  LightSample ls;
  ls.direction = Xyz4(light.axis_u);
  ls.distance = kFloatMax;
  ls.radiance = Xyz4(light.radiance);
  ls.pdf = 1.0f;
  ls.delta = true;
  return ls;
}

// CrossedLight (scene.slang:1019-1091).
F3 CrossedLight(const oracle_scene& s, uint32_t index, F3 origin, F3 direction, float distance, bool escaped,
    bool weigh, float pdf) {
  const AnalyticLight& light = s.analytic[index];
  float light_pdf = 0.0f;
  if (light.shape == kSphereLight) {
    const float radius = light.position[3];
    const F3 offset = origin - Xyz4(light.position);
    const float c = dot(offset, offset) - radius * radius;
    const float b = -dot(offset, direction);
    const F3 perpendicular = offset + b * direction;
    const float discriminant = radius * radius - dot(perpendicular, perpendicular);
    if (!(c > 0.0f) || !(b > 0.0f) || discriminant < 0.0f) return V(0.0f);
    const float t = c / (b + std::sqrt(discriminant));
    if (!(t < distance)) return V(0.0f);
    light_pdf = SphereConePdf(radius * radius / dot(offset, offset));
  } else if (light.shape == kRectLight || light.shape == kDiskLight) {
    const F3 n = Xyz4(light.normal);
    const float facing = dot(direction, n);
    if (!(facing < 0.0f)) return V(0.0f);
    const float t = dot(Xyz4(light.position) - origin, n) / facing;
    if (!(t > 0.0f) || !(t < distance)) return V(0.0f);
    const F3 q = origin + t * direction - Xyz4(light.position);
    const F3 u = Xyz4(light.axis_u), v = Xyz4(light.axis_v);
    const float uu = dot(u, u), uv = dot(u, v), vv = dot(v, v);
    const float qu = dot(q, u), qv = dot(q, v);
    const float determinant = uu * vv - uv * uv;
    const float a = (qu * vv - qv * uv) / determinant;
    const float b = (qv * uu - qu * uv) / determinant;
    if (light.shape == kRectLight ? !(std::fabs(a) <= 1.0f && std::fabs(b) <= 1.0f) : !(a * a + b * b <= 1.0f))
      return V(0.0f);
    light_pdf = t * t / (-facing * light.normal[3]);
  } else if (light.shape == kDistantLight && escaped) {
    const F3 toward = Xyz4(light.axis_u);
    const float one_minus_cos = light.axis_u[3];
    const float cosine = dot(direction, toward);
    if (one_minus_cos <= 1.0f) {
      const F3 across = cross(direction, toward);
      if (!(cosine > 0.0f) || !(dot(across, across) <= one_minus_cos * (2.0f - one_minus_cos))) return V(0.0f);
    } else if (!(cosine >= 1.0f - one_minus_cos)) {
      return V(0.0f);
    }
    light_pdf = 1.0f / (2.0f * kPi * one_minus_cos);
  } else {
    return V(0.0f);
  }
  const float weight = weigh ? PowerHeuristic(pdf, light.radiance[3] * light_pdf) : 1.0f;
  return Xyz4(light.radiance) * weight;
}

// OverlapsBox (scene.slang:1095-1103).
inline bool OverlapsBox(const float* low, const float* high, F3 origin, F3 inverse, float distance) {
  const float t0x = (low[0] - origin.x) * inverse.x, t1x = (high[0] - origin.x) * inverse.x;
  const float t0y = (low[1] - origin.y) * inverse.y, t1y = (high[1] - origin.y) * inverse.y;
  const float t0z = (low[2] - origin.z) * inverse.z, t1z = (high[2] - origin.z) * inverse.z;
  const float nx = std::fmin(t0x, t1x), ny = std::fmin(t0y, t1y), nz = std::fmin(t0z, t1z);
  const float fx = std::fmax(t0x, t1x), fy = std::fmax(t0y, t1y), fz = std::fmax(t0z, t1z);
  return std::fmax(std::fmax(nx, ny), std::fmax(nz, 0.0f)) <= std::fmin(std::fmin(fx, fy), std::fmin(fz, distance));
}

inline float SafeInverse(float d) {
  return 1.0f / (std::fabs(d) > 1e-30f ? d : (d < 0.0f ? -1e-30f : 1e-30f));
}

// CrossedLights (scene.slang:1110-1178): the crossing hierarchy's leaves in
// its traversal order, then, for an escaping ray, the distant lights.
F3 CrossedLights(const oracle_scene& s, F3 origin, F3 direction, float distance, bool escaped, bool weigh,
    float pdf) {
  F3 sum = V(0.0f);
  if (!s.light_nodes.empty()) {
    const F3 inverse = V(SafeInverse(direction.x), SafeInverse(direction.y), SafeInverse(direction.z));
    uint32_t stack[kLightStackSize];
    uint32_t depth = 0, node = 0;
    while (true) {
      const LightNode& current = s.light_nodes[node];
      const uint32_t child0 = AsUint(current.low0[3]);
      const uint32_t child1 = AsUint(current.low1[3]);
      const bool enter0 = OverlapsBox(current.low0, current.high0, origin, inverse, distance);
      const bool enter1 =
          child1 != kNoLightChild && OverlapsBox(current.low1, current.high1, origin, inverse, distance);
      uint32_t next = 0xFFFFFFFFu;
      if (enter0) {
        if ((child0 & kLightLeaf) != 0)
          sum = sum + CrossedLight(s, child0 & ~kLightLeaf, origin, direction, distance, escaped, weigh, pdf);
        else
          next = child0;
      }
      if (enter1) {
        if ((child1 & kLightLeaf) != 0)
          sum = sum + CrossedLight(s, child1 & ~kLightLeaf, origin, direction, distance, escaped, weigh, pdf);
        else if (next == 0xFFFFFFFFu)
          next = child1;
        else
          stack[depth++] = child1;
      }
      if (next == 0xFFFFFFFFu) {
        if (depth == 0) break;
        next = stack[--depth];
      }
      node = next;
    }
  }
  if (escaped)
    for (uint32_t index : s.distant)
      sum = sum + CrossedLight(s, index, origin, direction, distance, escaped, weigh, pdf);
  return sum;
}

// SampleLight (scene.slang:894-909).
LightSample SampleLight(const oracle_scene& s, const float* u, F3 origin) {
  const uint32_t count = static_cast<uint32_t>(s.lights.size());
  const uint32_t column = std::min(static_cast<uint32_t>(u[0] * float(count)), count - 1);
  const LightRecord& record = s.lights[column];
  const uint32_t light = u[1] < record.threshold ? column : record.alias;
  const LightRecord& chosen = s.lights[light];
  if (chosen.instance == kEnvironmentLight) return SampleEnvironment(s, chosen.pdf, u[2], u[3]);
  if ((chosen.instance & kAnalyticLight) != 0)
    return SampleAnalytic(s.analytic[chosen.instance & ~kAnalyticLight], chosen.pdf, u[2], u[3], origin);
  return SampleTriangle(s, light, chosen, u[2], u[3], origin);
}

// EmitterPdf (scene.slang:1004-1010).
float EmitterPdf(const oracle_scene& s, const Hit& hit, float area) {
  const uint32_t first = s.light_offsets[hit.instance];
  if (first == kNoLights || !(area > 0.0f)) return 0.0f;
  return s.lights[first + hit.primitive].pdf / area;
}

// ---------------------------------------------------------------------------
// transport.slang

struct PathState {
  Ray ray;
  F3 throughput;
  F3 radiance;
  uint32_t pixel_index;
  uint32_t depth;
  uint32_t rng;
  float last_pdf;
  uint32_t flags;
};
constexpr uint32_t kUnweightedLight = 1;

struct RestirRecord;  // below

struct FrameConstants {
  float clip_to_world[16];
  float ndc_from_pixel[4];
  uint32_t width;
  uint32_t max_bounces;
  bool sample_lights;
  // RestirInitial: the depth-0 direct light is the final reservoir's.
  const unsigned char* restir_final = nullptr;
  uint32_t restir_stride = 0;
};

struct RayCounts {
  uint64_t camera = 0, extension = 0, shadow = 0;
};

// CameraRay (scene.slang:273-283).
Ray CameraRay(const FrameConstants& f, float nx, float ny, float nz_far) {
  (void)nz_far;
  const float* c = f.clip_to_world;
  auto mul = [&](float x, float y, float z, float w, float* out) {
    for (int r = 0; r < 4; ++r)
      out[r] = c[r] * x + c[4 + r] * y + c[8 + r] * z + c[12 + r] * w;
  };
  float n[4], fa[4];
  mul(nx, ny, 0.0f, 1.0f, n);
  mul(nx, ny, 1.0f, 1.0f, fa);
  Ray ray;
  ray.origin = V(n[0] / n[3], n[1] / n[3], n[2] / n[3]);
  ray.direction = normalize(V(fa[0], fa[1], fa[2]) * n[3] - V(n[0], n[1], n[2]) * fa[3]);
  ray.tmin = 0.0f;
  ray.tmax = fa[3] == 0.0f ? kFloatMax
                           : length(V(fa[0] / fa[3], fa[1] / fa[3], fa[2] / fa[3]) - ray.origin);
  return ray;
}

// StartPath (transport.slang:53-69).
PathState StartPath(const FrameConstants& f, uint32_t px, uint32_t py, uint32_t sample_index) {
  PathState p;
  p.throughput = V(1.0f);
  p.radiance = V(0.0f);
  p.pixel_index = py * f.width + px;
  p.depth = 0;
  p.rng = SeedRandom(p.pixel_index, sample_index);
  p.last_pdf = 0.0f;
  p.flags = 0;
  const float ux = NextRandom(p.rng);
  const float uy = NextRandom(p.rng);
  const float film_x = float(px) + 0.5f + (ux - 0.5f);
  const float film_y = float(py) + 0.5f + (uy - 0.5f);
  p.ray = CameraRay(f, film_x * f.ndc_from_pixel[0] + f.ndc_from_pixel[2],
      film_y * f.ndc_from_pixel[1] + f.ndc_from_pixel[3], 1.0f);
  return p;
}

inline bool WeighFoundLight(const FrameConstants& f, const PathState& p) {
  return f.sample_lights && (p.flags & kUnweightedLight) == 0;
}

// ShadowedLight (transport.slang:82-115).
F3 ShadowedLight(const oracle_scene& s, const SurfaceHit& sh, const ShadingFrame& basis, F3 wo,
    F3 origin, const LightSample& ls, RayCounts& rays) {
  if (!(ls.pdf > 0.0f) || MaxComponent(ls.radiance) <= 0.0f || dot(ls.direction, sh.normal) <= 0.0f)
    return V(0.0f);
  const F3 wi = basis.ToLocal(ls.direction);
  if (wi.z <= 0.0f) return V(0.0f);
  const F3 f = BsdfEvaluate(sh, wo, wi);
  if (MaxComponent(f) <= 0.0f) return V(0.0f);
  Ray shadow{origin, 0.0f, ls.direction, ls.distance};
  ++rays.shadow;
  const float transmittance = ShadowTransmittance(s, shadow);
  if (transmittance <= 0.0f) return V(0.0f);
  const float weight = ls.delta ? 1.0f : PowerHeuristic(ls.pdf, BsdfPdf(sh, wo, wi));
  const F3 contribution = f * ls.radiance * (transmittance * weight / ls.pdf);
  return IsFinite(contribution) ? contribution : V(0.0f);
}

// DirectLight (transport.slang:123-135).
F3 DirectLight(const oracle_scene& s, const SurfaceHit& sh, const ShadingFrame& basis, F3 wo,
    uint32_t& rng, RayCounts& rays) {
  if (s.lights.empty()) return V(0.0f);
  float u[4];
  u[0] = NextRandom(rng);
  u[1] = NextRandom(rng);
  u[2] = NextRandom(rng);
  u[3] = NextRandom(rng);
  const F3 origin = OffsetRayOrigin(sh.position, sh.normal);
  return ShadowedLight(s, sh, basis, wo, origin, SampleLight(s, u, origin), rays);
}

// The reservoir records (restir.slang:11-60; vulkan_backend.hpp:152-178).
struct Reservoir {
  uint32_t sample;
  float weight_sum;
  float selected_target;
  uint32_t candidate_count;
};
struct RestirRecord {
  Reservoir reservoir;
  float uv[2];
  float proposal;
  uint32_t flags;
  float contribution[4];
};
static_assert(sizeof(RestirRecord) == 48, "RestirPixel is 48 bytes");
constexpr uint32_t kNoReservoirSample = 0xFFFFFFFFu;

// ReconstructReservoirLight (scene.slang:939-967): a sphere light's
// candidates are points uniform over its whole area.
LightSample ReconstructReservoirLight(const oracle_scene& s, uint32_t index, float ux, float uy, F3 origin) {
  const LightRecord& chosen = s.lights[index];
  if (chosen.instance == kEnvironmentLight) return SampleEnvironment(s, chosen.pdf, ux, uy);
  if ((chosen.instance & kAnalyticLight) == 0) return SampleTriangle(s, index, chosen, ux, uy, origin);
  const AnalyticLight& light = s.analytic[chosen.instance & ~kAnalyticLight];
  if (light.shape != kSphereLight) return SampleAnalytic(light, chosen.pdf, ux, uy, origin);
  const float z = 1.0f - 2.0f * ux;
  const float radius_xy = std::sqrt(std::fmax(0.0f, 1.0f - z * z));
  const float phi = 2.0f * kPi * uy;
  float sn, cs;
  lsincos(phi, sn, cs);
  const F3 normal = V(radius_xy * cs, radius_xy * sn, z);
  const F3 toward = Xyz4(light.position) + light.position[3] * normal - origin;
  const float distance2 = dot(toward, toward);
  if (!(distance2 > 0.0f)) return NoLight();
  LightSample ls = NoLight();
  ls.distance = std::sqrt(distance2);
  ls.direction = toward / ls.distance;
  const float cosine = -dot(normal, ls.direction);
  if (!(cosine > 0.0f)) return NoLight();
  ls.radiance = Xyz4(light.radiance);
  ls.pdf = chosen.pdf * distance2 / (cosine * 4.0f * kPi * light.position[3] * light.position[3]);
  return ls;
}

// ReservoirPartitionPdf (scene.slang:973-983): a sphere light's reservoir
// sample weighed at the cone density SampleLight would have used.
float ReservoirPartitionPdf(const oracle_scene& s, uint32_t index, const LightSample& ls, F3 origin) {
  const LightRecord& chosen = s.lights[index];
  if ((chosen.instance & kAnalyticLight) != 0 && chosen.instance != kEnvironmentLight) {
    const AnalyticLight& light = s.analytic[chosen.instance & ~kAnalyticLight];
    if (light.shape == kSphereLight) {
      const F3 offset = Xyz4(light.position) - origin;
      return chosen.pdf * SphereConePdf(light.position[3] * light.position[3] / dot(offset, offset));
    }
  }
  return ls.pdf;
}

// InitialDirectLight (restir.slang:235-254).
F3 InitialDirectLight(const oracle_scene& s, const FrameConstants& f, uint32_t pixel, const SurfaceHit& sh,
    const ShadingFrame& basis, F3 wo) {
  RestirRecord sel;
  std::memcpy(&sel, f.restir_final + size_t{pixel} * f.restir_stride, sizeof(sel));
  if ((sel.flags & 2u) != 0 || !(sel.reservoir.weight_sum > 0.0f) || sel.reservoir.sample >= s.lights.size())
    return V(0.0f);
  const F3 origin = OffsetRayOrigin(sh.position, sh.normal);
  const LightSample ls = ReconstructReservoirLight(s, sel.reservoir.sample, sel.uv[0], sel.uv[1], origin);
  const F3 wi = basis.ToLocal(ls.direction);
  const float weight = ls.delta ? 1.0f
      : PowerHeuristic(ReservoirPartitionPdf(s, sel.reservoir.sample, ls, origin),
            wi.z > 0.0f ? BsdfPdf(sh, wo, wi) : 0.0f);
  return V(sel.contribution[0], sel.contribution[1], sel.contribution[2]) * weight;
}

// EmissionWeight (transport.slang:150-158).
float EmissionWeight(const oracle_scene& s, const PathState& p, const Hit& hit, const SurfaceHit& sh) {
  const float area_pdf = EmitterPdf(s, hit, sh.area);
  if (!(area_pdf > 0.0f)) return 1.0f;
  const F3 toward = sh.position - p.ray.origin;
  const float cosine = std::fabs(dot(sh.normal, p.ray.direction));
  return PowerHeuristic(p.last_pdf, area_pdf * dot(toward, toward) / cosine);
}

// ParallelLights (transport.slang:139-146): under BSDF sampling, each
// parallel light through its own shadow ray.
F3 ParallelLights(const oracle_scene& s, const SurfaceHit& sh, const ShadingFrame& basis, F3 wo,
    RayCounts& rays) {
  const F3 origin = OffsetRayOrigin(sh.position, sh.normal);
  F3 sum = V(0.0f);
  for (uint32_t index = 0; index < s.analytic.size(); ++index)
    sum = sum + ShadowedLight(s, sh, basis, wo, origin, ParallelLight(s, index), rays);
  return sum;
}

// ScatterPath (transport.slang:164-230).
bool ScatterPath(const oracle_scene& s, const FrameConstants& f, PathState& p, const Hit& hit,
    RayCounts& rays) {
  const SurfaceHit sh = ReconstructHit(s, hit, p.ray.direction);
  F3 emission = sh.emission;
  if (WeighFoundLight(f, p) && p.depth != 0 && MaxComponent(emission) > 0.0f)
    emission = emission * EmissionWeight(s, p, hit, sh);
  p.radiance = p.radiance + p.throughput * emission;
  if (p.depth != 0 && !s.analytic.empty())
    p.radiance = p.radiance + p.throughput * CrossedLights(s, p.ray.origin, p.ray.direction,
        dot(sh.position - p.ray.origin, p.ray.direction), false, WeighFoundLight(f, p), p.last_pdf);
  if (p.depth >= f.max_bounces) return false;
  if (p.depth >= kRouletteBounces) {
    const float survival = std::fmin(MaxComponent(p.throughput), kMaxSurvival);
    if (NextRandom(p.rng) >= survival) return false;
    p.throughput = p.throughput / survival;
  }
  const ShadingFrame basis = MakeShadingFrame(sh.shading_normal);
  const F3 wo = basis.ToLocal(-p.ray.direction);
  if (f.restir_final && p.depth == 0)
    p.radiance = p.radiance + p.throughput * InitialDirectLight(s, f, p.pixel_index, sh, basis, wo);
  else if (f.sample_lights)
    p.radiance = p.radiance + p.throughput * DirectLight(s, sh, basis, wo, p.rng, rays);
  else if (!s.analytic.empty())
    p.radiance = p.radiance + p.throughput * ParallelLights(s, sh, basis, wo, rays);
  F3 u;
  u.x = NextRandom(p.rng);
  u.y = NextRandom(p.rng);
  u.z = NextRandom(p.rng);
  BsdfSampleResult sample;
  if (!BsdfSample(sh, wo, u, sample)) return false;
  const F3 wi = normalize(basis.ToWorld(sample.wi));
  const float side = dot(wi, sh.normal);
  if (sample.transmitted ? side >= 0.0f : side <= 0.0f) return false;
  p.throughput = p.throughput * sample.weight;
  p.last_pdf = sample.pdf;
  if (sample.delta || sample.transmitted)
    p.flags |= kUnweightedLight;
  else
    p.flags &= ~kUnweightedLight;
  p.ray.origin = OffsetRayOrigin(sh.position, sample.transmitted ? -sh.normal : sh.normal);
  p.ray.direction = wi;
  p.ray.tmin = 0.0f;
  p.ray.tmax = kFloatMax;
  ++p.depth;
  return true;
}

// MissPath (transport.slang:235-247).
void MissPath(const oracle_scene& s, const FrameConstants& f, PathState& p) {
  F3 environment = s.environment_constant;
  if (s.env.bound)
    environment = environment + EnvironmentRadiance(s, p.ray.direction, WeighFoundLight(f, p), p.last_pdf);
  p.radiance = p.radiance + p.throughput * environment;
  if (!s.analytic.empty())
    p.radiance = p.radiance + p.throughput * CrossedLights(s, p.ray.origin, p.ray.direction, kFloatMax, true,
        WeighFoundLight(f, p), p.last_pdf);
}

// TracePath and the radiance pass's sample (path_trace.slang:279-287,
// 357-366): the radiance of one camera path, or false when it misses.
bool PathSample(const oracle_scene& s, const FrameConstants& f, uint32_t px, uint32_t py,
    uint32_t sample_index, F3& radiance, RayCounts& rays) {
  PathState p = StartPath(f, px, py, sample_index);
  Hit hit;
  ++rays.camera;
  if (!Trace(s, p.ray, p.rng, hit)) return false;
  while (ScatterPath(s, f, p, hit, rays)) {
    ++rays.extension;
    if (!Trace(s, p.ray, p.rng, hit)) {
      MissPath(s, f, p);
      break;
    }
  }
  radiance = p.radiance;
  return true;
}

// Invert (vulkan_backend.cpp:436-470): Gauss-Jordan in double with partial
// pivoting.
bool Invert4(const float* matrix, float* inverse) {
  double rows[4][8] = {};
  for (int row = 0; row < 4; ++row) {
    for (int column = 0; column < 4; ++column) {
      const float value = matrix[column * 4 + row];
      if (!std::isfinite(value)) return false;
      rows[row][column] = value;
    }
    rows[row][row + 4] = 1.0;
  }
  for (int column = 0; column < 4; ++column) {
    int pivot = column;
    for (int row = column + 1; row < 4; ++row)
      if (std::abs(rows[row][column]) > std::abs(rows[pivot][column])) pivot = row;
    if (rows[pivot][column] == 0.0) return false;
    for (int index = 0; index < 8; ++index) std::swap(rows[column][index], rows[pivot][index]);
    const double scale = rows[column][column];
    for (double& value : rows[column]) value /= scale;
    for (int row = 0; row < 4; ++row) {
      if (row == column) continue;
      const double factor = rows[row][column];
      for (int index = 0; index < 8; ++index) rows[row][index] -= factor * rows[column][index];
    }
  }
  for (int row = 0; row < 4; ++row) {
    for (int column = 0; column < 4; ++column) {
      const float value = static_cast<float>(rows[row][column + 4]);
      if (!std::isfinite(value)) return false;
      inverse[column * 4 + row] = value;
    }
  }
  return true;
}

// The frame's constants: VulkanWorldToClip (vulkan_internal.hpp:326-336),
// Invert, and the display viewport's ndc_from_pixel
// (vulkan_backend.cpp:2406-2412, 651-658).
bool MakeFrame(const lotus_frame_desc& d, FrameConstants& f, uint32_t rect[4]) {
  float vulkan[16];
  std::memcpy(vulkan, d.world_to_clip, sizeof(vulkan));
  for (int column = 0; column < 4; ++column) {
    const float y = d.world_to_clip[column * 4 + 1];
    const float z = d.world_to_clip[column * 4 + 2];
    const float w = d.world_to_clip[column * 4 + 3];
    vulkan[column * 4 + 1] = -y;
    vulkan[column * 4 + 2] = 0.5f * (z + w);
  }
  if (!Invert4(vulkan, f.clip_to_world)) return false;
  const lotus_target& t = d.target;
  float vx = 0.0f, vy = 0.0f, vw = float(t.width), vh = float(t.height);
  if (t.display_window[2] > 0.0f && t.display_window[3] > 0.0f) {
    vx = t.display_window[0];
    vy = t.display_window[1];
    vw = t.display_window[2];
    vh = t.display_window[3];
  }
  f.ndc_from_pixel[0] = 2.0f / vw;
  f.ndc_from_pixel[1] = 2.0f / vh;
  f.ndc_from_pixel[2] = -2.0f * vx / vw - 1.0f;
  f.ndc_from_pixel[3] = -2.0f * vy / vh - 1.0f;
  f.width = t.width;
  f.max_bounces = d.settings.max_bounces;
  f.sample_lights = d.settings.light_sampling != LOTUS_LIGHT_SAMPLING_BSDF;
  const int32_t* w = t.data_window;
  if (w[2] <= 0 || w[3] <= 0) {
    rect[0] = 0; rect[1] = 0; rect[2] = t.width; rect[3] = t.height;
  } else {
    const int64_t x0 = std::max<int64_t>(w[0], 0), y0 = std::max<int64_t>(w[1], 0);
    const int64_t x1 = std::min<int64_t>(int64_t{w[0]} + w[2], t.width);
    const int64_t y1 = std::min<int64_t>(int64_t{w[1]} + w[3], t.height);
    if (x1 <= x0 || y1 <= y0) {
      rect[0] = rect[1] = rect[2] = rect[3] = 0;
    } else {
      rect[0] = uint32_t(x0); rect[1] = uint32_t(y0);
      rect[2] = uint32_t(x1 - x0); rect[3] = uint32_t(y1 - y0);
    }
  }
  return true;
}

int ThreadCount(int32_t threads) {
#ifdef _OPENMP
  return threads > 0 ? threads : omp_get_max_threads();
#else
  (void)threads;
  return 1;
#endif
}

void SetError(char* error, size_t size, const std::string& message) {
  if (error && size) std::snprintf(error, size, "%s", message.c_str());
}

}  // namespace

extern "C" {

oracle_scene* oracle_scene_create(const lotus_scene_desc* d, char* error, size_t error_size) {
  if (!d) {
    SetError(error, error_size, "no scene");
    return nullptr;
  }
  auto s = std::make_unique<oracle_scene>();
  s->materials.assign(d->materials, d->materials + d->material_count);
  if (s->materials.empty()) {
    SetError(error, error_size, "the scene has no material");
    return nullptr;
  }
  s->geometries.resize(d->geometry_count);
  for (uint32_t gi = 0; gi < d->geometry_count; ++gi) {
    const lotus_geometry& src = d->geometries[gi];
    Geometry& g = s->geometries[gi];
    g.positions.resize(src.vertex_count);
    for (uint32_t v = 0; v < src.vertex_count; ++v)
      g.positions[v] = V(src.positions[3 * v], src.positions[3 * v + 1], src.positions[3 * v + 2]);
    g.triangles.assign(src.triangles, src.triangles + 3 * size_t{src.triangle_count});
    for (uint32_t idx : g.triangles) {
      if (idx >= src.vertex_count) {
        SetError(error, error_size, "a triangle indexes past its geometry's vertices");
        return nullptr;
      }
    }
    if (src.normals) {
      g.normals.resize(3 * size_t{src.triangle_count});
      for (size_t k = 0; k < g.normals.size(); ++k)
        g.normals[k] = V(src.normals[3 * k], src.normals[3 * k + 1], src.normals[3 * k + 2]);
    }
    if (src.color_sets && src.colors && src.color_counts) {
      const float* c = src.colors;
      for (uint32_t k = 0; k < src.color_sets; ++k) {
        std::vector<F3> set(src.color_counts[k]);
        for (F3& v : set) {
          v = V(c[0], c[1], c[2]);
          c += 3;
        }
        g.colors.push_back(std::move(set));
      }
    }
    if (src.texcoord_sets && src.texcoords) {
      g.texcoord_sets = src.texcoord_sets;
      g.texcoords.assign(src.texcoords, src.texcoords + 6 * size_t{src.texcoord_sets} * src.triangle_count);
    }
    std::vector<Box> boxes(src.triangle_count);
    for (uint32_t t = 0; t < src.triangle_count; ++t)
      for (int k = 0; k < 3; ++k) {
        const F3 p = g.positions[g.triangles[3 * t + k]];
        const float a[3] = {p.x, p.y, p.z};
        boxes[t].Grow(a);
      }
    g.bvh.Build(boxes);
  }
  s->instances.resize(d->instance_count);
  std::vector<Box> instance_boxes(d->instance_count);
  for (uint32_t ii = 0; ii < d->instance_count; ++ii) {
    const lotus_instance& src = d->instances[ii];
    Instance& inst = s->instances[ii];
    std::memcpy(inst.m, src.world_from_object, sizeof(inst.m));
    inst.geometry = src.geometry;
    inst.material = src.material;
    inst.texcoord_set = src.texcoord_set;
    inst.color_set = src.color_set;
    if (src.geometry >= d->geometry_count || src.material >= d->material_count) {
      SetError(error, error_size, "an instance names a missing geometry or material");
      return nullptr;
    }
    if (!InvertAffine(inst.m, inst.inv)) {
      SetError(error, error_size, "an instance transform is singular");
      return nullptr;
    }
    const Geometry& g = s->geometries[inst.geometry];
    Box world;
    if (!g.bvh.nodes.empty() && !g.triangles.empty()) {
      const Box& b = g.bvh.nodes[0].box;
      for (int corner = 0; corner < 8; ++corner) {
        const F3 c = V((corner & 1) ? b.hi[0] : b.lo[0], (corner & 2) ? b.hi[1] : b.lo[1],
            (corner & 4) ? b.hi[2] : b.lo[2]);
        const F3 w = TransformPoint(inst.m, c);
        const float a[3] = {w.x, w.y, w.z};
        world.Grow(a);
      }
      // Widen by a relative margin so that float rounding of the corner
      // transform cannot cull a hit.
      for (int a = 0; a < 3; ++a) {
        const float pad = 1e-6f * std::max(std::fabs(world.lo[a]), std::fabs(world.hi[a])) + 1e-7f;
        world.lo[a] -= pad;
        world.hi[a] += pad;
      }
    }
    inst.world = world;
    instance_boxes[ii] = world;
  }
  s->tlas.Build(instance_boxes);
  // Textures decoded to linear RGBA: sRGB codes through the inverse
  // transfer function (linear below 0.04045, the 2.4 power above, in double),
  // alpha and unorm codes / 255.
  float srgb[256];
  for (int v = 0; v < 256; ++v) {
    const double c = v / 255.0;
    srgb[v] = static_cast<float>(c <= 0.04045 ? c / 12.92 : std::pow((c + 0.055) / 1.055, 2.4));
  }
  s->textures.resize(d->texture_count);
  for (uint32_t i = 0; i < d->texture_count; ++i) {
    const lotus_texture& src = d->textures[i];
    Texture& t = s->textures[i];
    t.width = src.width;
    t.height = src.height;
    const size_t n = size_t{src.width} * src.height;
    t.rgba.resize(4 * n);
    if (src.format == LOTUS_TEXTURE_RGBA32_FLOAT) {
      const float* f = static_cast<const float*>(src.texels);
      std::copy(f, f + 4 * n, t.rgba.begin());
    } else {
      const uint8_t* b = static_cast<const uint8_t*>(src.texels);
      for (size_t k = 0; k < 4 * n; ++k)
        t.rgba[k] = (src.format == LOTUS_TEXTURE_RGBA8_SRGB && k % 4 != 3) ? srgb[b[k]]
                                                                          : static_cast<float>(b[k] / 255.0);
    }
  }
  s->inputs.assign(d->texture_inputs, d->texture_inputs + d->texture_input_count);
  s->environment_constant = V(d->environment_constant[0], d->environment_constant[1], d->environment_constant[2]);
  if (d->environment && d->environment->texels && d->environment->width && d->environment->height) {
    const lotus_environment& e = *d->environment;
    s->env.width = e.width;
    s->env.height = e.height;
    s->env.texels.assign(e.texels, e.texels + 4 * size_t{e.width} * e.height);
    s->env.scale = V(e.scale[0], e.scale[1], e.scale[2]);
    for (int r = 0; r < 3; ++r)
      s->env.rows[r] = V(e.environment_from_world[3 * r], e.environment_from_world[3 * r + 1],
          e.environment_from_world[3 * r + 2]);
    BuildEnvironmentDistribution(s->env);
  }
  if (d->light_count) {
    if (!d->lights) {
      SetError(error, error_size, "light_count without lights");
      return nullptr;
    }
    s->light_inputs.assign(d->lights, d->lights + d->light_count);
    for (const lotus_light& l : s->light_inputs) {
      bool finite = true;
      for (float v : l.world_from_light) finite = finite && std::isfinite(v);
      for (float v : l.radiance) finite = finite && std::isfinite(v);
      finite = finite && std::isfinite(l.radius) && std::isfinite(l.width) && std::isfinite(l.height) &&
          std::isfinite(l.angle);
      if (l.shape > LOTUS_LIGHT_DISTANT || !finite) {
        SetError(error, error_size, "an analytic light has an unknown shape or non-finite values");
        return nullptr;
      }
    }
  }
  BuildLightTable(*s);
  return s.release();
}

void oracle_scene_destroy(oracle_scene* scene) { delete scene; }

int32_t oracle_sample(const oracle_scene* s, const lotus_frame_desc* d, uint32_t sample_index,
    float* rgba, uint64_t* rays, int32_t threads) {
  FrameConstants f;
  uint32_t rect[4];
  if (!s || !d || !rgba || !MakeFrame(*d, f, rect)) return LOTUS_FAIL;
  const int64_t pixels = int64_t{rect[2]} * rect[3];
  std::atomic<uint64_t> camera{0}, extension{0}, shadow{0};
#pragma omp parallel num_threads(ThreadCount(threads))
  {
    RayCounts local;
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < pixels; ++i) {
      const uint32_t px = rect[0] + uint32_t(i % rect[2]);
      const uint32_t py = rect[1] + uint32_t(i / rect[2]);
      F3 radiance;
      float* out = rgba + 4 * (size_t{py} * d->target.width + px);
      if (PathSample(*s, f, px, py, sample_index, radiance, local)) {
        out[0] = radiance.x; out[1] = radiance.y; out[2] = radiance.z; out[3] = 1.0f;
      } else {
        out[0] = out[1] = out[2] = out[3] = 0.0f;
      }
    }
    camera += local.camera;
    extension += local.extension;
    shadow += local.shadow;
  }
  if (rays) {
    rays[0] = camera;
    rays[1] = extension;
    rays[2] = shadow;
  }
  return LOTUS_PASS;
}

int32_t oracle_accumulate(const oracle_scene* s, const lotus_frame_desc* d, uint32_t first_sample,
    uint32_t count, double* sums, uint64_t* rays, int32_t threads) {
  FrameConstants f;
  uint32_t rect[4];
  if (!s || !d || !sums || !MakeFrame(*d, f, rect)) return LOTUS_FAIL;
  const int64_t pixels = int64_t{rect[2]} * rect[3];
  std::atomic<uint64_t> camera{0}, extension{0}, shadow{0};
#pragma omp parallel num_threads(ThreadCount(threads))
  {
    RayCounts local;
#pragma omp for schedule(dynamic, 16)
    for (int64_t i = 0; i < pixels; ++i) {
      const uint32_t px = rect[0] + uint32_t(i % rect[2]);
      const uint32_t py = rect[1] + uint32_t(i / rect[2]);
      double* out = sums + 4 * (size_t{py} * d->target.width + px);
      for (uint32_t k = 0; k < count; ++k) {
        F3 radiance;
        if (PathSample(*s, f, px, py, first_sample + k, radiance, local)) {
          out[0] += radiance.x;
          out[1] += radiance.y;
          out[2] += radiance.z;
          out[3] += 1.0;
        }
      }
    }
    camera += local.camera;
    extension += local.extension;
    shadow += local.shadow;
  }
  if (rays) {
    rays[0] = camera;
    rays[1] = extension;
    rays[2] = shadow;
  }
  return LOTUS_PASS;
}

int64_t oracle_light_table(const oracle_scene* s, uint32_t* records, uint64_t record_capacity,
    uint32_t* offsets, uint64_t offset_capacity) {
  if (!s) return -1;
  const uint64_t n = s->lights.size();
  if (records)
    for (uint64_t i = 0; i < n && i < record_capacity; ++i) {
      records[4 * i] = AsUint(s->lights[i].pdf);
      records[4 * i + 1] = AsUint(s->lights[i].threshold);
      records[4 * i + 2] = s->lights[i].alias;
      records[4 * i + 3] = s->lights[i].instance;
    }
  if (offsets)
    for (uint64_t i = 0; i < s->light_offsets.size() && i < offset_capacity; ++i)
      offsets[i] = s->light_offsets[i];
  return static_cast<int64_t>(n);
}

int32_t oracle_traversal_stats(const oracle_scene* s, const lotus_frame_desc* d, uint32_t max_rays,
    double* nodes_per_ray, double* triangles_per_ray) {
  FrameConstants f;
  uint32_t rect[4];
  if (!s || !d || !MakeFrame(*d, f, rect)) return LOTUS_FAIL;
  const uint64_t pixels = uint64_t{rect[2]} * rect[3];
  const uint64_t n = std::min<uint64_t>(pixels, max_rays ? max_rays : pixels);
  Counters c;
  for (uint64_t k = 0; k < n; ++k) {
    const uint64_t i = n == pixels ? k : (k * pixels) / n;
    const uint32_t px = rect[0] + uint32_t(i % rect[2]);
    const uint32_t py = rect[1] + uint32_t(i / rect[2]);
    PathState p = StartPath(f, px, py, 0);
    Hit hit;
    Trace(*s, p.ray, p.rng, hit, &c);
  }
  if (nodes_per_ray) *nodes_per_ray = n ? double(c.nodes) / n : 0.0;
  if (triangles_per_ray) *triangles_per_ray = n ? double(c.triangles) / n : 0.0;
  return LOTUS_PASS;
}

}  // extern "C"

// ===========================================================================
// Temporal passes: the primary-surface metadata (temporal.slang:557-627) and
// the ReSTIR DI reservoir passes (restir.slang:163-491), restated on the CPU
// over the same records the CUDA kernels write.

namespace {

struct TemporalPixelO {
  float normal_depth[4];
  float motion_depth[4];
  uint64_t instance_id;
  uint64_t material_id;
  uint32_t flags, albedo, shading_normal, reserved;
};
static_assert(sizeof(TemporalPixelO) == 64, "TemporalPixel is 64 bytes");
struct ValidityO {
  uint32_t valid, rejection, previous_index, reserved;
};
struct RestirReuseO {
  RestirRecord pixel;
  float normalization;
  uint32_t supporting_candidates;
  uint32_t previous_index;
  uint32_t age;
};
static_assert(sizeof(RestirReuseO) == 64, "RestirReuse is 64 bytes");
struct RestirSurfaceO {
  float origin[4], normal[4], shading_normal[4], outgoing[4], base_alpha[4], dielectric_metallic[4],
      fresnel[4], model[4], extension[4];
  uint64_t instance_id, material_id;
};
static_assert(sizeof(RestirSurfaceO) == 160, "RestirSurface is 160 bytes");

inline void Mul4(const float* m, float x, float y, float z, float w, float* o) {
  for (int r = 0; r < 4; ++r) o[r] = m[r] * x + m[4 + r] * y + m[8 + r] * z + m[12 + r] * w;
}

inline bool Finite4(const float* v) {
  return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]) && std::isfinite(v[3]);
}


uint32_t PackAlbedo(F3 c) {
  const uint32_t x = static_cast<uint32_t>(std::rint(Saturate(c.x) * 255.0f));
  const uint32_t y = static_cast<uint32_t>(std::rint(Saturate(c.y) * 255.0f));
  const uint32_t z = static_cast<uint32_t>(std::rint(Saturate(c.z) * 255.0f));
  return x | (y << 8) | (z << 16);
}

// PackNormal (temporal.slang:111-117).
uint32_t PackNormal(F3 n) {
  const float s = std::fabs(n.x) + std::fabs(n.y) + std::fabs(n.z);
  float ex = n.x / s, ey = n.y / s;
  if (n.z < 0.0f) {
    const float ox = (1.0f - std::fabs(ey)) * (ex >= 0.0f ? 1.0f : -1.0f);
    const float oy = (1.0f - std::fabs(ex)) * (ey >= 0.0f ? 1.0f : -1.0f);
    ex = ox;
    ey = oy;
  }
  const int qx = static_cast<int>(std::rint(std::fmin(std::fmax(ex, -1.0f), 1.0f) * 32767.0f));
  const int qy = static_cast<int>(std::rint(std::fmin(std::fmax(ey, -1.0f), 1.0f) * 32767.0f));
  return (static_cast<uint32_t>(qx) & 0xffffu) | (static_cast<uint32_t>(qy) << 16);
}

struct TemporalIds {
  float previous[12];  // rows
  uint64_t instance_id, material_id;
  uint32_t flags;
};

std::vector<TemporalIds> ConvertIds(const oracle_scene& s, const lotus_temporal_instance* ids) {
  std::vector<TemporalIds> out(s.instances.size());
  for (size_t i = 0; i < out.size(); ++i) {
    const float* m = ids ? ids[i].previous_world_from_object : s.instances[i].m;
    for (int r = 0; r < 3; ++r) {
      out[i].previous[4 * r] = m[r];
      out[i].previous[4 * r + 1] = m[4 + r];
      out[i].previous[4 * r + 2] = m[8 + r];
      out[i].previous[4 * r + 3] = m[12 + r];
    }
    out[i].instance_id = ids ? ids[i].instance_id : i;
    out[i].material_id = ids ? ids[i].material_id : s.instances[i].material;
    out[i].flags = ids ? ids[i].flags : 6u;
  }
  return out;
}

inline F3 RowPoint(const float* r, F3 p) {
  return V(r[0] * p.x + r[1] * p.y + r[2] * p.z + r[3], r[4] * p.x + r[5] * p.y + r[6] * p.z + r[7],
      r[8] * p.x + r[9] * p.y + r[10] * p.z + r[11]);
}

// WriteTemporalSurface (temporal.slang:557-627).
TemporalPixelO TemporalSurface(const oracle_scene& s, const FrameConstants& f, const oracle_temporal& tc,
    const std::vector<TemporalIds>& ids, uint32_t px, uint32_t py) {
  TemporalPixelO o{};
  const uint32_t index = py * f.width + px;
  uint32_t rng = SeedRandom(index, 0);
  const float cx = float(px) + 0.5f, cy = float(py) + 0.5f;
  const Ray ray = CameraRay(f, cx * f.ndc_from_pixel[0] + f.ndc_from_pixel[2],
      cy * f.ndc_from_pixel[1] + f.ndc_from_pixel[3], 1.0f);
  Hit hit;
  if (!Trace(s, ray, rng, hit)) return o;
  const Instance& inst = s.instances[hit.instance];
  const Geometry& g = s.geometries[inst.geometry];
  const TemporalIds& id = ids[hit.instance];
  const uint32_t* tri = &g.triangles[3 * hit.primitive];
  const F3 p0 = g.positions[tri[0]], p1 = g.positions[tri[1]], p2 = g.positions[tri[2]];
  const F3 point = p0 + hit.b1 * (p1 - p0) + hit.b2 * (p2 - p0);
  const F3 world = TransformPoint(inst.m, point);
  float view[4];
  Mul4(tc.current_view, world.x, world.y, world.z, 1.0f, view);
  const F3 a = TransformPoint(inst.m, p0), b = TransformPoint(inst.m, p1), c = TransformPoint(inst.m, p2);
  F3 normal = normalize(cross(b - a, c - a));
  if (dot(normal, ray.direction) > 0.0f) normal = -normal;
  const float depth = -view[2] / view[3];
  if (!(Finite4(view) && IsFinite(normal) && view[3] > 0.0f && depth > 0.0f)) return o;
  o.normal_depth[0] = normal.x; o.normal_depth[1] = normal.y; o.normal_depth[2] = normal.z;
  o.normal_depth[3] = depth;
  o.instance_id = id.instance_id;
  o.material_id = id.material_id;
  o.flags = 1u | id.flags;
  const SurfaceHit sh = ReconstructHit(s, hit, ray.direction);
  const F3 albedo = sh.bsdf.transmission > 0.0f
      ? sh.base_color + sh.bsdf.transmission * (sh.bsdf.transmission_color - sh.base_color)
      : sh.base_color;
  o.albedo = PackAlbedo(albedo);
  o.shading_normal = PackNormal(sh.shading_normal);
  if (id.flags & 2u) {
    const F3 pw = RowPoint(id.previous, point);
    float pv[4], clip[4];
    Mul4(tc.previous_view, pw.x, pw.y, pw.z, 1.0f, pv);
    Mul4(tc.previous_world_to_clip, pw.x, pw.y, pw.z, 1.0f, clip);
    const float qx = clip[0] / clip[3], qy = clip[1] / clip[3], qz = clip[2] / clip[3];
    const float pd = -pv[2] / pv[3];
    const float ppx = tc.previous_display[0] + (qx * 0.5f + 0.5f) * tc.previous_display[2];
    const float ppy = tc.previous_display[1] + (qy * 0.5f + 0.5f) * tc.previous_display[3];
    const float bx = float(tc.previous_data[0]), by = float(tc.previous_data[1]);
    const float ex = bx + float(tc.previous_data[2]), ey = by + float(tc.previous_data[3]);
    if (Finite4(pv) && Finite4(clip) && std::isfinite(ppx) && std::isfinite(ppy) && std::isfinite(pd) &&
        pv[3] > 0.0f && clip[3] > 0.0f && pd > 0.0f && qz >= 0.0f && qz <= 1.0f && qx >= -1.0f &&
        qy >= -1.0f && qx < 1.0f && qy < 1.0f && ppx >= bx && ppy >= by && ppx < ex && ppy < ey) {
      o.motion_depth[0] = ppx - cx;
      o.motion_depth[1] = ppy - cy;
      o.motion_depth[2] = pd;
      o.motion_depth[3] = 1.0f;
    }
  }
  return o;
}

// Reservoir arithmetic in float (reservoir.slang:23-103).
bool StreamCandidate(Reservoir& r, uint32_t sample, float target, float proposal, float random, bool& selected) {
  selected = false;
  const bool valid_zero = r.weight_sum == 0.0f && r.sample == kNoReservoirSample && r.selected_target == 0.0f;
  const bool valid_positive = r.weight_sum > 0.0f && r.sample != kNoReservoirSample &&
      r.selected_target > 0.0f && r.candidate_count != 0;
  if (!std::isfinite(r.weight_sum) || !std::isfinite(r.selected_target) || !(valid_zero || valid_positive) ||
      !std::isfinite(target) || target < 0.0f || !std::isfinite(proposal) || proposal <= 0.0f ||
      !std::isfinite(random) || random < 0.0f || random >= 1.0f ||
      (target > 0.0f && sample == kNoReservoirSample) || r.candidate_count == 0xFFFFFFFFu)
    return false;
  const float weight = target / proposal;
  const float sum = r.weight_sum + weight;
  if (!std::isfinite(weight) || !std::isfinite(sum) || (target > 0.0f && weight == 0.0f)) return false;
  selected = weight > 0.0f && (r.weight_sum == 0.0f || random < weight / sum);
  r.weight_sum = sum;
  ++r.candidate_count;
  if (selected) {
    r.sample = sample;
    r.selected_target = target;
  }
  return true;
}

inline float Normalization(const Reservoir& r) {
  return r.weight_sum > 0.0f ? (r.weight_sum / float(r.candidate_count)) / r.selected_target : 0.0f;
}

inline float ReuseNormalization(const Reservoir& r, uint32_t supporting) {
  return r.weight_sum > 0.0f ? (r.weight_sum / float(supporting)) / r.selected_target : 0.0f;
}

bool MergeReevaluated(Reservoir& d, const Reservoir& src, float normalization, float target, uint32_t cap,
    float random, bool& selected) {
  selected = false;
  const uint32_t count = std::min(src.candidate_count, cap);
  const bool zero = src.weight_sum == 0.0f && src.sample == kNoReservoirSample && src.selected_target == 0.0f &&
      normalization == 0.0f && target == 0.0f;
  const bool positive = src.weight_sum > 0.0f && src.selected_target > 0.0f && src.sample != kNoReservoirSample &&
      src.candidate_count != 0 && normalization > 0.0f;
  const bool valid_destination = d.weight_sum == 0.0f
      ? d.sample == kNoReservoirSample && d.selected_target == 0.0f
      : d.weight_sum > 0.0f && d.selected_target > 0.0f && d.sample != kNoReservoirSample && d.candidate_count != 0;
  if (!valid_destination || !std::isfinite(d.weight_sum) || !std::isfinite(d.selected_target) ||
      !std::isfinite(src.weight_sum) || !std::isfinite(src.selected_target) || !(zero || positive) ||
      !std::isfinite(normalization) || !std::isfinite(target) || target < 0.0f || cap == 0 ||
      !std::isfinite(random) || random < 0.0f || random >= 1.0f || count > 0xFFFFFFFFu - d.candidate_count)
    return false;
  const float weight = (target * normalization) * float(count);
  const float sum = d.weight_sum + weight;
  if (!std::isfinite(weight) || !std::isfinite(sum) || (target > 0.0f && weight == 0.0f)) return false;
  selected = weight > 0.0f && (d.weight_sum == 0.0f || random < weight / sum);
  d.weight_sum = sum;
  d.candidate_count += count;
  if (selected) {
    d.sample = src.sample;
    d.selected_target = target;
  }
  return true;
}

// ChooseReservoirLight and ReservoirProposalPdf (scene.slang:915-937).
uint32_t ChooseReservoirLight(const oracle_scene& s, uint32_t proposal, float ux, float uy) {
  const uint32_t count = static_cast<uint32_t>(s.lights.size());
  const uint32_t column = std::min(static_cast<uint32_t>(ux * float(count)), count - 1);
  if (proposal == 1) return column;
  if (proposal == 2) {
    if (uy < 0.5f) return column;
    uy = (uy - 0.5f) * 2.0f;
  }
  const LightRecord& record = s.lights[column];
  return uy < record.threshold ? column : record.alias;
}

float ReservoirProposalPdf(const oracle_scene& s, uint32_t proposal, uint32_t index) {
  const float power = s.lights[index].pdf;
  const float uniform = 1.0f / float(s.lights.size());
  if (proposal == 1) return uniform;
  if (proposal == 2) return 0.5f * (power + uniform);
  return power;
}

// A stored surface's closure: its model's tag and representation
// (BsdfClosure, bsdf.slang:26-30).
struct StoredClosureO {
  bool gltf = false;
  PreviewClosure preview;
  ComposedClosure composed;
};

// ReflectionEvaluate (restir.slang:66-72).
inline F3 ReflectionEvaluate(const StoredClosureO& c, F3 wo, F3 wi) {
  if (!(wi.z > 0.0f)) return V(0.0f);
  return c.gltf ? ComposedEvaluate(c.composed, wo, wi) : PreviewEvaluate(c.preview, wo, wi);
}

// CandidateContribution (restir.slang:155-161).
F3 CandidateContribution(const SurfaceHit& sh, const ShadingFrame& basis, F3 wo, const LightSample& ls,
    float selection) {
  if (!(ls.pdf > 0.0f) || dot(ls.direction, sh.normal) <= 0.0f) return V(0.0f);
  const F3 wi = basis.ToLocal(ls.direction);
  const F3 f = wi.z > 0.0f ? BsdfEvaluate(sh, wo, wi) : V(0.0f);
  return f * ls.radiance * (selection / ls.pdf);
}

// PackGltfPbrTerms (gltf_pbr.slang:162-188).
void PackGltfPbrTerms(const GltfPbrTerms& g, float lanes[22]) {
  lanes[0] = g.base_color.x; lanes[1] = g.base_color.y; lanes[2] = g.base_color.z;
  lanes[3] = g.alpha; lanes[4] = g.metallic; lanes[5] = g.e1; lanes[6] = g.share;
  lanes[7] = g.f0.x; lanes[8] = g.f0.y; lanes[9] = g.f0.z; lanes[10] = g.f90;
  lanes[11] = g.transmission; lanes[12] = g.coat_scale; lanes[13] = g.coat_dim; lanes[14] = g.coat_alpha;
  lanes[15] = g.coat_normal.x; lanes[16] = g.coat_normal.y;
  lanes[17] = g.sheen_color.x; lanes[18] = g.sheen_color.y; lanes[19] = g.sheen_color.z;
  lanes[20] = g.sheen_roughness; lanes[21] = g.sheen_dim;
}

// UnpackGltfPbrTerms (gltf_pbr.slang:190-214).
GltfPbrTerms UnpackGltfPbrTerms(const float lanes[22]) {
  GltfPbrTerms g;
  g.base_color = V(lanes[0], lanes[1], lanes[2]);
  g.alpha = lanes[3];
  g.metallic = lanes[4];
  g.e1 = lanes[5];
  g.share = lanes[6];
  g.f0 = V(lanes[7], lanes[8], lanes[9]);
  g.f90 = lanes[10];
  g.transmission = lanes[11];
  g.coat_scale = lanes[12];
  g.coat_dim = lanes[13];
  g.coat_alpha = lanes[14];
  const float tx = lanes[15], ty = lanes[16];
  g.coat_normal = V(tx, ty, std::sqrt(std::fmax(1.0f - (tx * tx + ty * ty), 0.0f)));
  g.sheen_color = V(lanes[17], lanes[18], lanes[19]);
  g.sheen_roughness = lanes[20];
  g.sheen_dim = lanes[21];
  return g;
}

// StoreClosure / LoadClosure (restir.slang:78-149).
void StoreClosure(const SurfaceHit& sh, RestirSurfaceO& o) {
  for (int k = 0; k < 4; ++k) o.model[k] = o.extension[k] = 0.0f;
  if (sh.gltf) {
    float lanes[22];
    PackGltfPbrTerms(sh.gltf_terms, lanes);
    o.model[0] = 1.0f;
    o.base_alpha[0] = lanes[0]; o.base_alpha[1] = lanes[1]; o.base_alpha[2] = lanes[2]; o.base_alpha[3] = lanes[3];
    o.dielectric_metallic[0] = lanes[7]; o.dielectric_metallic[1] = lanes[8];
    o.dielectric_metallic[2] = lanes[9]; o.dielectric_metallic[3] = lanes[4];
    o.model[1] = lanes[5]; o.model[2] = lanes[6]; o.model[3] = lanes[10];
    o.normal[3] = lanes[11];
    o.shading_normal[3] = lanes[12];
    o.outgoing[3] = lanes[13];
    o.fresnel[0] = lanes[14]; o.fresnel[1] = lanes[15]; o.fresnel[2] = lanes[16]; o.fresnel[3] = lanes[20];
    o.extension[0] = lanes[17]; o.extension[1] = lanes[18]; o.extension[2] = lanes[19]; o.extension[3] = lanes[21];
    return;
  }
  const PreviewClosure& b = sh.bsdf;
  o.normal[3] = b.dielectric_f90;
  o.shading_normal[3] = b.thin_walled ? -b.transmission : b.transmission;
  o.outgoing[3] = b.smooth ? -b.eta : b.eta;
  o.base_alpha[0] = b.base_color.x; o.base_alpha[1] = b.base_color.y; o.base_alpha[2] = b.base_color.z;
  o.base_alpha[3] = b.alpha;
  o.dielectric_metallic[0] = b.dielectric_f0.x; o.dielectric_metallic[1] = b.dielectric_f0.y;
  o.dielectric_metallic[2] = b.dielectric_f0.z; o.dielectric_metallic[3] = b.metallic;
  o.fresnel[0] = b.f0.x; o.fresnel[1] = b.f0.y; o.fresnel[2] = b.f0.z; o.fresnel[3] = b.f90;
}

StoredClosureO LoadClosure(const RestirSurfaceO& o) {
  StoredClosureO c;
  if ((uint32_t)o.model[0] == 1u) {
    float lanes[22];
    lanes[0] = o.base_alpha[0]; lanes[1] = o.base_alpha[1]; lanes[2] = o.base_alpha[2]; lanes[3] = o.base_alpha[3];
    lanes[4] = o.dielectric_metallic[3];
    lanes[5] = o.model[1]; lanes[6] = o.model[2];
    lanes[7] = o.dielectric_metallic[0]; lanes[8] = o.dielectric_metallic[1]; lanes[9] = o.dielectric_metallic[2];
    lanes[10] = o.model[3];
    lanes[11] = o.normal[3];
    lanes[12] = o.shading_normal[3];
    lanes[13] = o.outgoing[3];
    lanes[14] = o.fresnel[0]; lanes[15] = o.fresnel[1]; lanes[16] = o.fresnel[2];
    lanes[17] = o.extension[0]; lanes[18] = o.extension[1]; lanes[19] = o.extension[2];
    lanes[20] = o.fresnel[3];
    lanes[21] = o.extension[3];
    c.gltf = true;
    c.composed = MakeGltfPbrClosure(UnpackGltfPbrTerms(lanes), V(o.outgoing[0], o.outgoing[1], o.outgoing[2]));
    return c;
  }
  PreviewClosure& b = c.preview;
  b.base_color = V(o.base_alpha[0], o.base_alpha[1], o.base_alpha[2]);
  b.alpha = o.base_alpha[3];
  b.metallic = o.dielectric_metallic[3];
  b.dielectric_f0 = V(o.dielectric_metallic[0], o.dielectric_metallic[1], o.dielectric_metallic[2]);
  b.dielectric_f90 = o.normal[3];
  b.f0 = V(o.fresnel[0], o.fresnel[1], o.fresnel[2]);
  b.f90 = o.fresnel[3];
  b.transmission = std::fabs(o.shading_normal[3]);
  b.transmission_color = V(1.0f);
  b.eta = std::fabs(o.outgoing[3]);
  b.thin_walled = o.shading_normal[3] < 0.0f;
  b.smooth = o.outgoing[3] < 0.0f;
  return c;
}

inline F3 Xyz(const float* v) { return V(v[0], v[1], v[2]); }

// HistoryContribution (restir.slang:256-268).
F3 HistoryContribution(const oracle_scene& s, const RestirSurfaceO& src, uint32_t light, const LightSample& ls) {
  if (!(ls.pdf > 0.0f) || dot(ls.direction, Xyz(src.normal)) <= 0.0f) return V(0.0f);
  const StoredClosureO b = LoadClosure(src);
  const ShadingFrame basis = MakeShadingFrame(Xyz(src.shading_normal));
  return ReflectionEvaluate(b, Xyz(src.outgoing), basis.ToLocal(ls.direction)) * ls.radiance *
      (s.lights[light].pdf / ls.pdf);
}

F3 HistoryContributionUv(const oracle_scene& s, const RestirSurfaceO& src, uint32_t light, const float* uv) {
  return HistoryContribution(s, src, light, ReconstructReservoirLight(s, light, uv[0], uv[1], Xyz(src.origin)));
}

inline bool SameSample(const RestirRecord& a, const RestirRecord& b) {
  return a.reservoir.sample == b.reservoir.sample && a.uv[0] == b.uv[0] && a.uv[1] == b.uv[1];
}

float HistoryTarget(const oracle_scene& s, const RestirReuseO& source, const RestirSurfaceO& surface,
    const RestirRecord& selected, bool& valid) {
  if (SameSample(source.pixel, selected)) {
    valid = std::isfinite(source.pixel.reservoir.selected_target);
    return source.pixel.reservoir.selected_target;
  }
  const F3 c = HistoryContributionUv(s, surface, selected.reservoir.sample, selected.uv);
  valid = IsFinite(c);
  return MaxComponent(c);
}

float ReceiverVisibility(const oracle_scene& s, const RestirRecord& selected, const RestirRecord& current,
    F3 origin, const LightSample& ls) {
  if (SameSample(selected, current)) return current.contribution[3];
  return ShadowTransmittance(s, Ray{origin, 0.0f, ls.direction, ls.distance});
}

RestirRecord EmptyRecord() {
  RestirRecord r{};
  r.reservoir.sample = kNoReservoirSample;
  return r;
}

inline bool InRect(const uint32_t* rect, uint32_t px, uint32_t py) {
  return px >= rect[0] && py >= rect[1] && px < rect[0] + rect[2] && py < rect[1] + rect[3];
}

inline void SetContribution(RestirRecord& r, F3 e, float visibility) {
  r.contribution[0] = e.x; r.contribution[1] = e.y; r.contribution[2] = e.z; r.contribution[3] = visibility;
}

// WriteInitialReservoir (restir.slang:163-233).
RestirRecord InitialReservoir(const oracle_scene& s, const FrameConstants& f, const oracle_temporal& tc,
    const uint32_t* rect, uint32_t sample_index, uint32_t px, uint32_t py) {
  RestirRecord r = EmptyRecord();
  const uint32_t slot = py * f.width + px;
  if (!(tc.restir_candidates != 0 && InRect(rect, px, py))) return r;
  PathState p = StartPath(f, px, py, sample_index);
  Hit hit;
  if (!Trace(s, p.ray, p.rng, hit)) return r;
  r.flags |= 1u;
  const SurfaceHit sh = ReconstructHit(s, hit, p.ray.direction);
  const ShadingFrame basis = MakeShadingFrame(sh.shading_normal);
  const F3 wo = basis.ToLocal(-p.ray.direction);
  const F3 origin = OffsetRayOrigin(sh.position, sh.normal);
  uint32_t rng = SeedRandom(slot, sample_index ^ 0xD1B54A35u);
  if (tc.max_bounces != 0 && !s.lights.empty()) {
    for (uint32_t i = 0; i < tc.restir_candidates; ++i) {
      const float cx = NextRandom(rng);
      const float cy = NextRandom(rng);
      const float ux = NextRandom(rng);
      const float uy = NextRandom(rng);
      const float random = NextRandom(rng);
      const uint32_t light = ChooseReservoirLight(s, tc.restir_proposal, cx, cy);
      const float proposal = ReservoirProposalPdf(s, tc.restir_proposal, light);
      const LightSample ls = ReconstructReservoirLight(s, light, ux, uy, origin);
      const F3 fc = CandidateContribution(sh, basis, wo, ls, s.lights[light].pdf);
      bool selected;
      if (!std::isfinite(ls.pdf) || !IsFinite(fc) ||
          !StreamCandidate(r.reservoir, light, MaxComponent(fc), proposal, random, selected)) {
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
    const LightSample ls = ReconstructReservoirLight(s, r.reservoir.sample, r.uv[0], r.uv[1], origin);
    const float visibility = ShadowTransmittance(s, Ray{origin, 0.0f, ls.direction, ls.distance});
    const float normalization = Normalization(r.reservoir);
    const F3 estimate = CandidateContribution(sh, basis, wo, ls, s.lights[r.reservoir.sample].pdf) *
        (visibility * normalization);
    if (!std::isfinite(normalization) || !IsFinite(estimate))
      r.flags |= 2u;
    else
      SetContribution(r, estimate, visibility);
  }
  return r;
}

// WriteTemporalReservoir (restir.slang:302-387).
void TemporalReservoir(const oracle_scene& s, const FrameConstants& f, const oracle_temporal& tc,
    const uint32_t* rect, uint32_t sample_index, const std::vector<TemporalIds>& ids,
    const RestirRecord* initial, const ValidityO* validity, const TemporalPixelO* surface,
    const RestirReuseO* previous, const RestirSurfaceO* previous_surfaces, uint32_t px, uint32_t py,
    RestirReuseO& result, RestirSurfaceO& receiver) {
  const uint32_t slot = py * f.width + px;
  result = RestirReuseO{};
  receiver = RestirSurfaceO{};
  result.pixel = initial[slot];
  result.previous_index = 0xffffffffu;
  result.normalization = Normalization(result.pixel.reservoir);
  result.supporting_candidates = result.pixel.reservoir.candidate_count;
  if (!(tc.restir_candidates != 0 && InRect(rect, px, py))) return;
  PathState p = StartPath(f, px, py, sample_index);
  Hit hit;
  if (!Trace(s, p.ray, p.rng, hit)) return;
  const SurfaceHit sh = ReconstructHit(s, hit, p.ray.direction);
  const ShadingFrame basis = MakeShadingFrame(sh.shading_normal);
  const F3 wo = basis.ToLocal(-p.ray.direction);
  const F3 origin = OffsetRayOrigin(sh.position, sh.normal);
  float view[4];
  Mul4(tc.current_view, sh.position.x, sh.position.y, sh.position.z, 1.0f, view);
  receiver.origin[0] = origin.x; receiver.origin[1] = origin.y; receiver.origin[2] = origin.z;
  receiver.origin[3] = -view[2] / view[3];
  receiver.normal[0] = sh.normal.x; receiver.normal[1] = sh.normal.y; receiver.normal[2] = sh.normal.z;
  receiver.shading_normal[0] = sh.shading_normal.x; receiver.shading_normal[1] = sh.shading_normal.y;
  receiver.shading_normal[2] = sh.shading_normal.z;
  receiver.outgoing[0] = wo.x; receiver.outgoing[1] = wo.y; receiver.outgoing[2] = wo.z;
  StoreClosure(sh, receiver);
  receiver.instance_id = ids[hit.instance].instance_id;
  receiver.material_id = ids[hit.instance].material_id;
  const ValidityO v = validity[slot];
  const uint32_t previous_index = v.previous_index;
  const bool history = v.valid != 0 && surface[slot].instance_id == receiver.instance_id &&
      surface[slot].material_id == receiver.material_id;
  if (tc.restir_history != 0 && (result.pixel.flags & 2u) == 0 && history) {
    const RestirReuseO source = previous[previous_index];
    const RestirSurfaceO& psrc = previous_surfaces[previous_index];
    if ((source.pixel.flags & 1u) != 0 && (source.pixel.flags & 2u) == 0 &&
        psrc.instance_id == receiver.instance_id && psrc.material_id == receiver.material_id) {
      const uint32_t count = std::min(source.pixel.reservoir.candidate_count, tc.restir_max_history);
      F3 received = V(0.0f);
      if (source.pixel.reservoir.weight_sum > 0.0f) {
        if (source.pixel.reservoir.sample >= s.lights.size())
          result.pixel.flags |= 2u;
        else
          received = HistoryContributionUv(s, receiver, source.pixel.reservoir.sample, source.pixel.uv);
      }
      uint32_t rng = SeedRandom(slot, sample_index ^ 0x94D049BBu);
      bool selected;
      if (!IsFinite(received) || (result.pixel.flags & 2u) != 0 ||
          !MergeReevaluated(result.pixel.reservoir, source.pixel.reservoir, source.normalization,
              MaxComponent(received), tc.restir_max_history, NextRandom(rng), selected)) {
        result.pixel.flags |= 2u;
      } else {
        result.previous_index = previous_index;
        if (selected) {
          result.pixel.uv[0] = source.pixel.uv[0];
          result.pixel.uv[1] = source.pixel.uv[1];
          result.pixel.proposal = source.pixel.proposal;
          result.age = std::min(source.age, 65535u) + 1u;
        }
        if (result.pixel.reservoir.weight_sum > 0.0f) {
          bool valid_support;
          const float support = HistoryTarget(s, source, psrc, result.pixel, valid_support);
          if (!valid_support) result.pixel.flags |= 2u;
          result.supporting_candidates = initial[slot].reservoir.candidate_count + (support > 0.0f ? count : 0u);
        } else {
          result.supporting_candidates = 0;
        }
        result.normalization = ReuseNormalization(result.pixel.reservoir, result.supporting_candidates);
      }
    }
  }
  if ((result.pixel.flags & 2u) == 0 && result.pixel.reservoir.weight_sum > 0.0f) {
    const LightSample ls = ReconstructReservoirLight(s, result.pixel.reservoir.sample, result.pixel.uv[0],
        result.pixel.uv[1], origin);
    const float visibility = ReceiverVisibility(s, result.pixel, initial[slot], origin, ls);
    const F3 estimate = HistoryContribution(s, receiver, result.pixel.reservoir.sample, ls) *
        (visibility * result.normalization);
    if (!std::isfinite(result.normalization) || result.normalization <= 0.0f || !IsFinite(estimate))
      result.pixel.flags |= 2u;
    else
      SetContribution(result.pixel, estimate, visibility);
  }
}

// SpatialCompatible and WriteSpatialReservoir (restir.slang:392-491).
bool SpatialCompatible(const RestirSurfaceO& receiver, const RestirReuseO& record, const RestirSurfaceO& source) {
  return (record.pixel.flags & 3u) == 1u && receiver.origin[3] > 0.0f && source.origin[3] > 0.0f &&
      receiver.material_id == source.material_id &&
      std::fabs(receiver.origin[3] - source.origin[3]) <=
          0.01f + 0.02f * std::fmax(receiver.origin[3], source.origin[3]) &&
      dot(Xyz(receiver.normal), Xyz(source.normal)) >= 0.9f &&
      dot(Xyz(receiver.shading_normal), Xyz(source.shading_normal)) >= 0.9f;
}

// The spatial pass's neighbour offsets (the CUDA kernel's spatial_offsets):
// the reference's four axis neighbours at the radius (restir.slang:408-410),
// or, an extension of the reference, `count` distinct offsets drawn
// uniformly from the disk of the radius without its centre, each the first
// of up to 16 draws in the enclosing square that falls inside the disk and
// was not drawn before, from the stream seeded with sample_index ^
// 0x5BD1E995.
constexpr int kMaxNeighbours = 8;

int SpatialOffsets(uint32_t slot, uint32_t sample_index, int radius, uint32_t count, int* ox, int* oy) {
  if (count == 0) {
    const int ax[4] = {-radius, radius, 0, 0};
    const int ay[4] = {0, 0, -radius, radius};
    for (int i = 0; i < 4; ++i) ox[i] = ax[i], oy[i] = ay[i];
    return 4;
  }
  uint32_t rng = SeedRandom(slot, sample_index ^ 0x5BD1E995u);
  const float side = static_cast<float>(2 * radius + 1);
  int n = 0;
  for (uint32_t i = 0; i < count; ++i) {
    for (int t = 0; t < 16; ++t) {
      const int dx = std::min(static_cast<int>(NextRandom(rng) * side), 2 * radius) - radius;
      const int dy = std::min(static_cast<int>(NextRandom(rng) * side), 2 * radius) - radius;
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

void SpatialReservoirAll(const oracle_scene& s, const FrameConstants& f, const oracle_temporal& tc, uint32_t height,
    uint32_t sample_index, const RestirReuseO* temporal, const RestirSurfaceO* surfaces, uint32_t px, uint32_t py,
    RestirReuseO& result, uint32_t* sources) {
  const uint32_t slot = py * f.width + px;
  const RestirReuseO centre = temporal[slot];
  const RestirSurfaceO& receiver = surfaces[slot];
  result = centre;
  for (int i = 0; i < kMaxNeighbours; ++i) sources[i] = 0xffffffffu;
  if ((centre.pixel.flags & 3u) != 1u) return;
  int ox[kMaxNeighbours], oy[kMaxNeighbours];
  const int neighbours =
      SpatialOffsets(slot, sample_index, static_cast<int>(tc.restir_radius), tc.restir_neighbours, ox, oy);
  uint32_t accepted = 0;
  for (int i = 0; i < neighbours; ++i) {
    const int nx = static_cast<int>(px) + ox[i], ny = static_cast<int>(py) + oy[i];
    if (nx < 0 || ny < 0 || nx >= static_cast<int>(f.width) || ny >= static_cast<int>(height)) continue;
    const uint32_t index = static_cast<uint32_t>(ny) * f.width + static_cast<uint32_t>(nx);
    if (SpatialCompatible(receiver, temporal[index], surfaces[index])) {
      sources[i] = index;
      ++accepted;
    }
  }
  if (accepted == 0) return;
  result.pixel.reservoir = Reservoir{kNoReservoirSample, 0.0f, 0.0f, 0};
  bool selected;
  if (!MergeReevaluated(result.pixel.reservoir, centre.pixel.reservoir, centre.normalization,
          centre.pixel.reservoir.selected_target, 0xffffffffu, 0.0f, selected))
    result.pixel.flags |= 2u;
  uint32_t rng = SeedRandom(slot, sample_index ^ 0x369DEA0Fu);
  for (int i = 0; i < neighbours; ++i) {
    if (sources[i] == 0xffffffffu) continue;
    const RestirReuseO& source = temporal[sources[i]];
    F3 received = V(0.0f);
    if (source.pixel.reservoir.weight_sum > 0.0f)
      received = HistoryContributionUv(s, receiver, source.pixel.reservoir.sample, source.pixel.uv);
    if (!IsFinite(received) ||
        !MergeReevaluated(result.pixel.reservoir, source.pixel.reservoir, source.normalization,
            MaxComponent(received), tc.restir_max_history, NextRandom(rng), selected)) {
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
  for (int k = 0; k < 4; ++k) result.pixel.contribution[k] = 0.0f;
  if ((result.pixel.flags & 2u) == 0 && result.pixel.reservoir.weight_sum > 0.0f) {
    result.supporting_candidates = centre.pixel.reservoir.candidate_count;
    for (int i = 0; i < neighbours; ++i) {
      if (sources[i] == 0xffffffffu) continue;
      const RestirReuseO& source = temporal[sources[i]];
      bool valid_support;
      const float support = HistoryTarget(s, source, surfaces[sources[i]], result.pixel, valid_support);
      if (!valid_support) result.pixel.flags |= 2u;
      if (support > 0.0f)
        result.supporting_candidates += std::min(source.pixel.reservoir.candidate_count, tc.restir_max_history);
    }
  }
  result.normalization = ReuseNormalization(result.pixel.reservoir, result.supporting_candidates);
  if ((result.pixel.flags & 2u) == 0 && result.pixel.reservoir.weight_sum > 0.0f) {
    const LightSample ls = ReconstructReservoirLight(s, result.pixel.reservoir.sample, result.pixel.uv[0],
        result.pixel.uv[1], Xyz(receiver.origin));
    const float visibility = ReceiverVisibility(s, result.pixel, centre.pixel, Xyz(receiver.origin), ls);
    const F3 estimate = HistoryContribution(s, receiver, result.pixel.reservoir.sample, ls) *
        (visibility * result.normalization);
    if (!std::isfinite(result.normalization) || result.normalization <= 0.0f || !IsFinite(estimate))
      result.pixel.flags |= 2u;
    else
      SetContribution(result.pixel, estimate, visibility);
  }
}

// SpatialReservoirAll with the first four sources kept (the product's
// layout: the reference's four axis neighbours).
void SpatialReservoir(const oracle_scene& s, const FrameConstants& f, const oracle_temporal& tc, uint32_t height,
    uint32_t sample_index, const RestirReuseO* temporal, const RestirSurfaceO* surfaces, uint32_t px, uint32_t py,
    RestirReuseO& result, uint32_t* sources) {
  uint32_t all[kMaxNeighbours];
  SpatialReservoirAll(s, f, tc, height, sample_index, temporal, surfaces, px, py, result, all);
  for (int i = 0; i < 4; ++i) sources[i] = all[i];
}

}  // namespace

extern "C" {

int32_t oracle_temporal_surface(const oracle_scene* s, const lotus_frame_desc* d, const oracle_temporal* tc,
    const lotus_temporal_instance* ids, void* out) {
  FrameConstants f;
  uint32_t rect[4];
  if (!s || !d || !tc || !out || !MakeFrame(*d, f, rect)) return LOTUS_FAIL;
  const auto identities = ConvertIds(*s, ids);
  auto* o = static_cast<TemporalPixelO*>(out);
  const int64_t n = int64_t{d->target.width} * d->target.height;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    const uint32_t px = uint32_t(i % d->target.width), py = uint32_t(i / d->target.width);
    o[i] = InRect(rect, px, py) ? TemporalSurface(*s, f, *tc, identities, px, py) : TemporalPixelO{};
  }
  return LOTUS_PASS;
}

int32_t oracle_restir_initial(const oracle_scene* s, const lotus_frame_desc* d, const oracle_temporal* tc,
    uint32_t sample_index, void* out) {
  FrameConstants f;
  uint32_t rect[4];
  if (!s || !d || !tc || !out || !MakeFrame(*d, f, rect)) return LOTUS_FAIL;
  auto* o = static_cast<RestirRecord*>(out);
  const int64_t n = int64_t{d->target.width} * d->target.height;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i)
    o[i] = InitialReservoir(*s, f, *tc, rect, sample_index, uint32_t(i % d->target.width),
        uint32_t(i / d->target.width));
  return LOTUS_PASS;
}

int32_t oracle_restir_temporal(const oracle_scene* s, const lotus_frame_desc* d, const oracle_temporal* tc,
    const lotus_temporal_instance* ids, uint32_t sample_index, const void* initial, const void* validity,
    const void* surface, const void* previous, const void* previous_surfaces, void* out, void* out_surfaces) {
  FrameConstants f;
  uint32_t rect[4];
  if (!s || !d || !tc || !MakeFrame(*d, f, rect)) return LOTUS_FAIL;
  const auto identities = ConvertIds(*s, ids);
  const int64_t n = int64_t{d->target.width} * d->target.height;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i)
    TemporalReservoir(*s, f, *tc, rect, sample_index, identities, static_cast<const RestirRecord*>(initial),
        static_cast<const ValidityO*>(validity), static_cast<const TemporalPixelO*>(surface),
        static_cast<const RestirReuseO*>(previous), static_cast<const RestirSurfaceO*>(previous_surfaces),
        uint32_t(i % d->target.width), uint32_t(i / d->target.width), static_cast<RestirReuseO*>(out)[i],
        static_cast<RestirSurfaceO*>(out_surfaces)[i]);
  return LOTUS_PASS;
}

int32_t oracle_restir_spatial(const oracle_scene* s, const lotus_frame_desc* d, const oracle_temporal* tc,
    uint32_t sample_index, const void* temporal, const void* surfaces, void* out, uint32_t* sources) {
  FrameConstants f;
  uint32_t rect[4];
  if (!s || !d || !tc || !MakeFrame(*d, f, rect)) return LOTUS_FAIL;
  const int64_t n = int64_t{d->target.width} * d->target.height;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i)
    SpatialReservoir(*s, f, *tc, d->target.height, sample_index, static_cast<const RestirReuseO*>(temporal),
        static_cast<const RestirSurfaceO*>(surfaces), uint32_t(i % d->target.width),
        uint32_t(i / d->target.width), static_cast<RestirReuseO*>(out)[i], sources + 4 * i);
  return LOTUS_PASS;
}

int32_t oracle_sample_restir(const oracle_scene* s, const lotus_frame_desc* d, uint32_t sample_index,
    const void* final_records, uint32_t stride, float* rgba, uint64_t* rays, int32_t threads) {
  FrameConstants f;
  uint32_t rect[4];
  if (!s || !d || !rgba || !final_records || !MakeFrame(*d, f, rect)) return LOTUS_FAIL;
  f.sample_lights = true;
  f.restir_final = static_cast<const unsigned char*>(final_records);
  f.restir_stride = stride;
  const int64_t pixels = int64_t{rect[2]} * rect[3];
  std::atomic<uint64_t> camera{0}, extension{0}, shadow{0};
#pragma omp parallel num_threads(ThreadCount(threads))
  {
    RayCounts local;
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < pixels; ++i) {
      const uint32_t px = rect[0] + uint32_t(i % rect[2]);
      const uint32_t py = rect[1] + uint32_t(i / rect[2]);
      F3 radiance;
      float* out = rgba + 4 * (size_t{py} * d->target.width + px);
      if (PathSample(*s, f, px, py, sample_index, radiance, local)) {
        out[0] = radiance.x; out[1] = radiance.y; out[2] = radiance.z; out[3] = 1.0f;
      } else {
        out[0] = out[1] = out[2] = out[3] = 0.0f;
      }
    }
    camera += local.camera;
    extension += local.extension;
    shadow += local.shadow;
  }
  if (rays) {
    rays[0] = camera;
    rays[1] = extension;
    rays[2] = shadow;
  }
  return LOTUS_PASS;
}

}  // extern "C"
