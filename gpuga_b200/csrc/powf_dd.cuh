// x^y for the Tersoff bond order in FP32 with a double-float exponent.
//
// The bond order b = (1 + zeta^n)^(-1/(2n)) needs x^y to about one unit in
// the last place: fr - b fa cancels near equilibrium, so a relative error in b
// reaches the site energy amplified.  Forming exp2(y * log2(x)) with FP32
// intermediates is not enough (the product y * log2(x) carries |y log2 x| *
// 2^-24 of absolute error into the exponent), so log2(x) and the product are
// kept as unevaluated sums hi + lo of two floats:
//
//   x = 2^e m, m in [sqrt(1/2), sqrt(2)),  f = m - 1 (exact),
//   s = f / (2 + f) as s_h + s_l (reciprocal estimate, exact FMA residual),
//   log2(m) = (2/ln 2) atanh(s) = K (s + s^3/3 + s^5/5 + ... + s^9/9),  |s| <= 0.1716
//     (the omitted terms: below K s^11 / 11 < 1.1e-9 absolute),
//   L = e + log2(m) (Fast2Sum: |e| >= 1 > |log2 m| or e = 0),
//   t = y L (exact FMA residual),  2^t = 2^k 2^r, k = rint(t_h), |r| <= 1/2,
//   2^r = sum_{i<=7} (r ln 2)^i / i!  (Taylor series; truncation < 6e-9 relative).
//
// The series are the Taylor expansions of atanh and of exp; the double-float
// steps are Dekker's exact product (via FMA) and Fast2Sum.  Domain: x > 0
// (the bond order only raises zeta >= 1e-16 and 1 + zeta^n); NaN x returns
// NaN, x = +inf and |y log2 x| > 125 give +inf or 0 (results below 2^-125
// flush to zero), zero and subnormal x give 0 for y > 0.  Negative x is not
// accepted.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#ifndef __CUDACC__
#define GPUGA_HD inline
#else
#define GPUGA_HD __host__ __device__ __forceinline__
#endif

namespace gpuga {

GPUGA_HD float pdd_as_float(int32_t i) {
#ifdef __CUDA_ARCH__
  return __int_as_float(i);
#else
  float f;
  std::memcpy(&f, &i, 4);
  return f;
#endif
}

GPUGA_HD int32_t pdd_as_int(float f) {
#ifdef __CUDA_ARCH__
  return __float_as_int(f);
#else
  int32_t i;
  std::memcpy(&i, &f, 4);
  return i;
#endif
}

GPUGA_HD float pdd_rcp(float t) {
#ifdef __CUDA_ARCH__
  return __fdividef(1.0f, t);  // estimate; the residual step below makes s exact to ~2^-46
#else
  return 1.0f / t;
#endif
}

// LO: the exponent carries a remainder, y + y_lo (the two- and three-argument forms below).
template <bool LO>
GPUGA_HD float powf_dd_t(float x, float y, float y_lo) {
#ifndef __CUDA_ARCH__
  if (x != x) return x;  // NaN (on the device: selected at the end, without a branch)
#endif
  // x = 2^e m with m in [sqrt(1/2), sqrt(2))
  const int32_t ix = pdd_as_int(x);
  const int32_t e = (ix - 0x3f3504f3) >> 23;
  const float m = pdd_as_float((int32_t)((uint32_t)ix - ((uint32_t)e << 23)));
  const float f = m - 1.0f;  // exact
  // s = f / (2 + f) as s_h + s_l; t_lo recovers the bit 2 + f may lose
  const float t = 2.0f + f;
  const float t_lo = (2.0f - t) + f;
  const float rc = pdd_rcp(t);
  const float s_h = f * rc;
  float res = fmaf(-s_h, t, f);
  res = fmaf(-s_h, t_lo, res);
  const float s_l = res * rc;
  // log2(m) = K s + K s^3 (1/3 + s^2/5 + s^4/7 + s^6/9), K = 2/ln 2 = K_h + K_l
  const float K_h = 2.885390043258667f, K_l = 3.851926067000022e-08f;
  const float s2 = s_h * s_h;
  float p = fmaf(s2, 1.0f / 9.0f, 1.0f / 7.0f);
  p = fmaf(s2, p, 1.0f / 5.0f);
  p = fmaf(s2, p, 1.0f / 3.0f);
  const float q = s_h * s2 * p;
  const float l_h = K_h * s_h;
  float l_l = fmaf(K_h, s_h, -l_h);  // exact error of the product
  l_l = fmaf(K_l, s_h, l_l);
  l_l = fmaf(K_h, s_l, l_l);
  l_l = fmaf(K_h, q, l_l);
  // L = e + log2(m): Fast2Sum (|e| >= 1 > |l_h|, or e = 0)
  const float ef = (float)e;
  const float L_h = ef + l_h;
  const float L_l = ((ef - L_h) + l_h) + l_l;
  // t = y L
  const float t_h = y * L_h;
  float t_l = fmaf(y, L_h, -t_h);
  t_l = fmaf(y, L_l, t_l);
  if (LO) t_l = fmaf(y_lo, L_h, t_l);  // y = y + y_lo when the exponent itself is a rounded FP64 value
  // 2^t = 2^k 2^r (out of range: selected away at the end, no branch)
  const float k = rintf(t_h);
  const float r = (t_h - k) + t_l;
  float u = fmaf(r, 1.5252733804059838e-05f, 1.5403530393381606e-04f);
  u = fmaf(r, u, 1.3333558146428441e-03f);
  u = fmaf(r, u, 9.618129107628477e-03f);
  u = fmaf(r, u, 5.5504108664821576e-02f);
  u = fmaf(r, u, 2.402265069591007e-01f);
  u = fmaf(r, u, 6.931471805599453e-01f);
  const float p2 = fmaf(r, u, 1.0f);
  const float v = pdd_as_float(pdd_as_int(p2) + (int32_t)k * (1 << 23));
  const float out = fabsf(t_h) <= 125.0f ? v : (t_h > 0.0f ? INFINITY : 0.0f);
#ifdef __CUDA_ARCH__
  return x != x ? x : out;
#else
  return out;
#endif
}

GPUGA_HD float powf_dd(float x, float y) { return powf_dd_t<false>(x, y, 0.0f); }
GPUGA_HD float powf_dd(float x, float y, float y_lo) { return powf_dd_t<true>(x, y, y_lo); }

}  // namespace gpuga
