// SPDX-License-Identifier: Apache-2.0
// The transport's elementary functions: sine and cosine, arctangent and
// arccosine, and the fifth power, written out so that the device and any
// host that evaluates the same operation sequence in FP32 without fused
// multiply-adds get bit-identical results. The reference leaves their
// precision to the shading language (Slang's sin, cos, atan2, acos and pow,
// whose SPIR-V precision is implementation-defined).
//
// sin/cos: Cody and Waite's range reduction ("Software Manual for the
// Elementary Functions", 1980) by pi/2 split into three floats (the first
// two with trailing zero bits, so k * P1 and k * P2 are exact for |k| <
// 2^11), then the Taylor polynomials of sin and cos on [-pi/4, pi/4],
// truncated after the x^9 and x^10 terms (remainders below 3e-9).
// atan: one argument reduction atan(a) = pi/4 + atan((a - 1)/(a + 1)) for
// a in (tan(pi/8), 1], then the Taylor series to t^21 (remainder below
// 1e-10 for |t| <= tan(pi/8)). acos(x) = atan2(sqrt((1 - x)(1 + x)), x).
#pragma once

#if defined(__CUDACC__)
#include <cuda_runtime.h>
#endif

#include <cmath>
#include <cstdint>
#include <cstring>

namespace lotus {

#if defined(__CUDACC__)
#define LOTUS_HD __host__ __device__ __forceinline__
#else
#define LOTUS_HD inline
#endif

LOTUS_HD void lsincos(float x, float& s, float& c) {
  const float k = rintf(x * 0.636619772f);
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

LOTUS_HD float lsin(float x) {
  float s, c;
  lsincos(x, s, c);
  return s;
}

LOTUS_HD float lcos(float x) {
  float s, c;
  lsincos(x, s, c);
  return c;
}

// atan(a) for a in [0, 1].
LOTUS_HD float latan_unit(float a) {
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

LOTUS_HD float latan2(float y, float x) {
  const float ax = fabsf(x), ay = fabsf(y);
  const float mx = ax > ay ? ax : ay;
  const float mn = ax > ay ? ay : ax;
  if (mx == 0.0f) return x < 0.0f ? (y < 0.0f ? -3.14159274f : 3.14159274f) : 0.0f;
  float r = latan_unit(mn / mx);
  if (ay > ax) r = 1.57079637f - r;
  if (x < 0.0f) r = 3.14159274f - r;
  return y < 0.0f ? -r : r;
}

// For x in [-1, 1].
LOTUS_HD float lacos(float x) { return latan2(sqrtf((1.0f - x) * (1.0f + x)), x); }

// pow(x, 5) as products.
LOTUS_HD float lpow5(float x) {
  const float x2 = x * x;
  return x2 * x2 * x;
}

LOTUS_HD uint32_t lbits(float x) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(x);
#else
  uint32_t u;
  memcpy(&u, &x, sizeof(u));
  return u;
#endif
}

LOTUS_HD float lfloat(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float x;
  memcpy(&x, &u, sizeof(x));
  return x;
#endif
}

// Natural logarithm for finite x > 0 (-infinity at 0, NaN below). The
// argument is split as m * 2^e with m in [sqrt(1/2), sqrt(2)), and
// log(m) = 2 atanh(s), s = (m - 1) / (m + 1), |s| <= 0.1716, by its
// series to s^15 (remainder below 1e-13); e * log(2) is added in two
// parts, the first exact for |e| < 2^9.
LOTUS_HD float llog(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? -lfloat(0x7f800000u) : lfloat(0x7fc00000u);
  int e = 0;
  if (x < 1.17549435e-38f) {
    x *= 8388608.0f;  // 2^23: a subnormal becomes normal
    e = -23;
  }
  const uint32_t b = lbits(x);
  e += (int)((b >> 23) & 0xffu) - 127;
  float m = lfloat((b & 0x7fffffu) | 0x3f800000u);
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

// e^x: x = k log(2) + r with |r| <= log(2)/2 (Cody and Waite's reduction,
// log(2) in the same two parts as above), e^r by its Taylor series to r^8
// (remainder below 4e-9 relative), times 2^k assembled from bits.
LOTUS_HD float lexp(float x) {
  if (!(x > -104.0f)) return x == x ? 0.0f : x;
  if (x > 89.0f) return lfloat(0x7f800000u);
  const float k = rintf(x * 1.44269502f);
  const float r = (x - k * 0.693145751953125f) - k * 1.42860677e-6f;
  const float p = 1.0f + r * (1.0f + r * (0.5f + r * (0.166666672f + r * (0.0416666679f +
      r * (0.00833333377f + r * (0.00138888892f + r * (0.000198412701f + r * 2.48015876e-5f)))))));
  int ki = (int)k;
  float scale = 1.0f;
  if (ki < -126) {
    ki += 64;
    scale = 5.42101086e-20f;  // 2^-64
  } else if (ki > 127) {
    ki -= 1;
    scale = 2.0f;
  }
  return p * lfloat((uint32_t)(ki + 127) << 23) * scale;
}

// x^y for x >= 0 and y > 0.
LOTUS_HD float lpow(float x, float y) {
  return x > 0.0f ? lexp(y * llog(x)) : 0.0f;
}

}  // namespace lotus
