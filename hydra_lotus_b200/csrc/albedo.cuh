// SPDX-License-Identifier: Apache-2.0
// Directional albedo tables of the composed closure's GGX and sheen lobes
// (backend/vulkan/shaders/bsdf/albedo.slang in hydra-lotus): E1, GGX
// reflection with a Fresnel of 1; Eschlick, the same with (1 - cos)^5; the
// rough dielectric's reflected albedo on three sheets (entering, leaving
// with total internal reflection, thin wall) over 16 relative indices; and
// the sheen's albedo. Each table is a grid over coordinates in [0, 1] read
// by Catmull-Rom splines along every axis. The grid's axes, node counts and
// layout follow albedo.slang exactly, so the data means the same thing; the
// values themselves come from albedo_tables_gen.cpp's own quadrature of the
// lobes in this library.
//
// The functions are host and device: the table generator checks its
// interpolation through them, and the renderer reads the uploaded data.
#pragma once

#include <cstdint>

#include "lmath.cuh"

namespace lotus {
namespace albedo {

constexpr uint32_t kGgx = 0;
constexpr uint32_t kSchlickShare = 1;
constexpr uint32_t kDielectric = 2;
constexpr uint32_t kSheen = 3;
constexpr uint32_t kTables = 4;

constexpr uint32_t kEntering = 0;
constexpr uint32_t kLeaving = 1;
constexpr uint32_t kThin = 2;
constexpr uint32_t kSheets = 3;

constexpr uint32_t kGgxCosines = 32;
constexpr uint32_t kDielectricCosines = 48;
constexpr uint32_t kAlphas = 32;
constexpr uint32_t kIndices = 16;

constexpr float kMinIndex = 1.01f;
constexpr float kMaxIndex = 3.0f;
constexpr float kMinCosine = 2.0e-4f;
constexpr float kCosineSlope = 4.0f;
constexpr float kAlphaSlope = 2.0f;
constexpr float kIndexSlope = 0.5f;
constexpr float kMinAlphaAxis = 1.0e-3f;
constexpr float kMinSheenAxis = 0.005f;
constexpr uint32_t kCriticalNode = kDielectricCosines / 2;
constexpr float kCriticalCoordinate = float(kCriticalNode) / float(kDielectricCosines - 1);
constexpr float kMinEvanescent = 2.0e-3f;

LOTUS_HD constexpr uint32_t cosines(uint32_t table) {
  return table == kDielectric ? kDielectricCosines : kGgxCosines;
}

// The first float of a table; offset(kTables) is the data's size.
LOTUS_HD constexpr uint32_t offset(uint32_t table) {
  return table <= kDielectric ? table * kGgxCosines * kAlphas
                              : (table - 1) * kGgxCosines * kAlphas +
                                kSheets * kIndices * kDielectricCosines * kAlphas;
}

constexpr uint32_t kSize = offset(kTables);
static_assert(kSize == 76800, "albedo table layout");

LOTUS_HD float unit_clamp(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }

// log(v) + slope * v over [low, high], normalized to [0, 1].
LOTUS_HD float log_linear(float v, float slope) { return llog(v) + slope * v; }

LOTUS_HD float log_linear_coordinate(float v, float low, float high, float slope) {
  const float c = fminf(fmaxf(v, low), high);
  return (log_linear(c, slope) - log_linear(low, slope)) /
      (log_linear(high, slope) - log_linear(low, slope));
}

LOTUS_HD float cosine_coordinate(float c) {
  return log_linear_coordinate(c, kMinCosine, 1.0f, kCosineSlope);
}
LOTUS_HD float alpha_coordinate(float a) {
  return log_linear_coordinate(a, kMinAlphaAxis, 1.0f, kAlphaSlope);
}
LOTUS_HD float sheen_coordinate(float r) {
  return log_linear_coordinate(r, kMinSheenAxis, 1.0f, kAlphaSlope);
}
LOTUS_HD float index_coordinate(float index) {
  return log_linear_coordinate(index - 1.0f, kMinIndex - 1.0f, kMaxIndex - 1.0f, kIndexSlope);
}

// The cosine at which a denser medium of relative index `index` reflects
// totally.
LOTUS_HD float critical_cosine(float index) {
  return sqrtf(fmaxf(1.0f - 1.0f / (index * index), 0.0f));
}

// Below the critical angle: log(mu) - log(tau) + slope mu, tau the
// evanescent cosine eta sqrt(mu_c^2 - mu^2), floored.
LOTUS_HD float evanescent_scale(float mu, float index, float critical) {
  const float tau = fmaxf(index * sqrtf(fmaxf(critical * critical - mu * mu, 0.0f)), kMinEvanescent);
  return llog(mu) - llog(tau) + kCosineSlope * mu;
}

// The leaving sheet's cosine coordinate: the nodes up to kCriticalNode span
// [kMinCosine, critical], those above it the refracted cosine's axis.
LOTUS_HD float leaving_coordinate(float c, float index) {
  const float critical = critical_cosine(index);
  if (c < critical) {
    const float low = evanescent_scale(kMinCosine, index, critical);
    const float high = evanescent_scale(critical, index, critical);
    return kCriticalCoordinate *
        unit_clamp((evanescent_scale(fmaxf(c, kMinCosine), index, critical) - low) / (high - low));
  }
  const float refracted = sqrtf(fmaxf(1.0f - index * index * (1.0f - c * c), 0.0f));
  const float x = cosine_coordinate(refracted);
  return kCriticalCoordinate + (1.0f - kCriticalCoordinate) * x;
}

// Catmull-Rom weights of the four nodes about a fraction t of a cell.
struct Cubic {
  float w[4];
};

LOTUS_HD Cubic cubic_weights(float t) {
  const float t2 = t * t;
  const float t3 = t2 * t;
  Cubic c;
  c.w[0] = -0.5f * t3 + t2 - 0.5f * t;
  c.w[1] = 1.5f * t3 - 2.5f * t2 + 1.0f;
  c.w[2] = -1.5f * t3 + 2.0f * t2 + 0.5f * t;
  c.w[3] = 0.5f * t3 - 0.5f * t2;
  return c;
}

// A node of a cosines x kAlphas slice; nodes beyond [first, last] along the
// cosine, or beyond the alpha axis, are extrapolated linearly from the two
// nearest inside.
LOTUS_HD float fetch_node(const float* __restrict__ t, uint32_t base, int n_cos, int c, int a,
    int first, int last) {
  const int last_a = (int)kAlphas - 1;
  const int cc = c < first ? first : (c > last ? last : c);
  const int ac = a < 0 ? 0 : (a > last_a ? last_a : a);
  const int dc = c < first ? 1 : (c > last ? -1 : 0);
  const int da = a < 0 ? 1 : (a > last_a ? -1 : 0);
  const float at = t[base + (uint32_t)(ac * n_cos + cc)];
  if (dc == 0 && da == 0) return at;
  const float inner = t[base + (uint32_t)((ac + da) * n_cos + cc + dc)];
  return 2.0f * at - inner;
}

// A slice's value at coordinates (x_cos, x_alpha); with `split` the cosine
// nodes on either side of kCriticalNode are separate pieces.
LOTUS_HD float fetch_slice(const float* __restrict__ t, uint32_t base, uint32_t n_cos, float x_cos,
    float x_alpha, bool split) {
  const float fc = unit_clamp(x_cos) * (float)(n_cos - 1);
  const float fa = unit_clamp(x_alpha) * (float)(kAlphas - 1);
  const uint32_t ic = (uint32_t)fc, ia = (uint32_t)fa;
  const int c0 = (int)(ic < n_cos - 2 ? ic : n_cos - 2);
  const int a0 = (int)(ia < kAlphas - 2 ? ia : kAlphas - 2);
  int first = 0, last = (int)n_cos - 1;
  if (split) {
    if (c0 < (int)kCriticalNode) last = (int)kCriticalNode;
    else first = (int)kCriticalNode;
  }
  const Cubic wc = cubic_weights(fc - (float)c0);
  const Cubic wa = cubic_weights(fa - (float)a0);
  float value = 0.0f;
  for (int j = 0; j < 4; ++j) {
    float row = 0.0f;
    for (int i = 0; i < 4; ++i)
      row += wc.w[i] * fetch_node(t, base, (int)n_cos, c0 + i - 1, a0 + j - 1, first, last);
    value += wa.w[j] * row;
  }
  return value;
}

// E1 at the outgoing cosine and GGX alpha.
LOTUS_HD float ggx(const float* __restrict__ t, float cos_theta, float alpha) {
  return fetch_slice(t, offset(kGgx), kGgxCosines, cosine_coordinate(cos_theta),
      alpha_coordinate(alpha), false);
}

// E1 and Eschlick at one (cosine, alpha): the two tables share their grid,
// so one pass computes the coordinates, weights and node indices once and
// reads both. Each value equals the one-table lookup's bit for bit.
LOTUS_HD void ggx_and_share(const float* __restrict__ t, float cos_theta, float alpha, float& e1,
    float& share) {
  constexpr uint32_t n_cos = kGgxCosines;
  const float fc = unit_clamp(cosine_coordinate(cos_theta)) * (float)(n_cos - 1);
  const float fa = unit_clamp(alpha_coordinate(alpha)) * (float)(kAlphas - 1);
  const uint32_t ic = (uint32_t)fc, ia = (uint32_t)fa;
  const int c0 = (int)(ic < n_cos - 2 ? ic : n_cos - 2);
  const int a0 = (int)(ia < kAlphas - 2 ? ia : kAlphas - 2);
  const Cubic wc = cubic_weights(fc - (float)c0);
  const Cubic wa = cubic_weights(fa - (float)a0);
  float v0 = 0.0f, v1 = 0.0f;
  for (int j = 0; j < 4; ++j) {
    float r0 = 0.0f, r1 = 0.0f;
    for (int i = 0; i < 4; ++i) {
      r0 += wc.w[i] * fetch_node(t, offset(kGgx), (int)n_cos, c0 + i - 1, a0 + j - 1, 0, (int)n_cos - 1);
      r1 += wc.w[i] * fetch_node(t, offset(kSchlickShare), (int)n_cos, c0 + i - 1, a0 + j - 1, 0, (int)n_cos - 1);
    }
    v0 += wa.w[j] * r0;
    v1 += wa.w[j] * r1;
  }
  e1 = v0;
  share = v1;
}

// Eschlick: the albedo per unit (f90 - f0) of Schlick's Fresnel.
LOTUS_HD float schlick_share(const float* __restrict__ t, float cos_theta, float alpha) {
  return fetch_slice(t, offset(kSchlickShare), kGgxCosines, cosine_coordinate(cos_theta),
      alpha_coordinate(alpha), false);
}

// The sheen's albedo for a white colour; above 1 toward grazing outgoing
// directions at small roughness.
LOTUS_HD float sheen(const float* __restrict__ t, float cos_theta, float roughness) {
  return fmaxf(fetch_slice(t, offset(kSheen), kGgxCosines, cosine_coordinate(cos_theta),
      sheen_coordinate(roughness), false), 0.0f);
}

// A rough dielectric's reflected albedo at relative index eta from the
// outgoing side, total internal reflection included.
LOTUS_HD float dielectric(const float* __restrict__ t, float cos_theta, float alpha, float eta,
    bool thin_walled) {
  uint32_t sheet = thin_walled ? kThin : kEntering;
  float index = eta;
  if (eta < 1.0f) {
    index = 1.0f / eta;
    sheet = thin_walled ? kThin : kLeaving;
  }
  index = fminf(fmaxf(index, kMinIndex), kMaxIndex);
  const float fi = index_coordinate(index) * (float)(kIndices - 1);
  const uint32_t ii = (uint32_t)fi;
  const int i0 = (int)(ii < kIndices - 2 ? ii : kIndices - 2);
  const bool split = sheet == kLeaving;
  const float x_cos = split ? leaving_coordinate(cos_theta, index) : cosine_coordinate(cos_theta);
  const float x_alpha = alpha_coordinate(alpha);
  const uint32_t slice_size = kDielectricCosines * kAlphas;
  const uint32_t base = offset(kDielectric) + sheet * kIndices * slice_size;
  float s[4];
  for (int j = 0; j < 4; ++j) {
    int k = i0 + j - 1;
    k = k < 0 ? 0 : (k > (int)kIndices - 1 ? (int)kIndices - 1 : k);
    s[j] = fetch_slice(t, base + (uint32_t)k * slice_size, kDielectricCosines, x_cos, x_alpha, split);
  }
  if (i0 == 0) s[0] = 2.0f * s[1] - s[2];
  if (i0 == (int)kIndices - 2) s[3] = 2.0f * s[2] - s[1];
  const Cubic w = cubic_weights(fi - (float)i0);
  return w.w[0] * s[0] + w.w[1] * s[1] + w.w[2] * s[2] + w.w[3] * s[3];
}

}  // namespace albedo
}  // namespace lotus
