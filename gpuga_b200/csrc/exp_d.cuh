// e^x in FP64 for the Tersoff pair terms, written for this engine.
//
// The batched Tersoff kernels evaluate fr = cr e^{-lr t} and fa = ca e^{-la t} in FP64
// (their difference cancels near equilibrium).  A general-purpose FP64 exponential carries
// a slow path for arguments near the overflow and underflow limits whose registers made the
// force kernel spill; this one has no branch:
//
//   k = round(x / ln 2), taken from the low mantissa bits of x log2(e) + 1.5 * 2^52
//       (adding the shifter rounds the product to an integer in round-to-nearest mode);
//   r = x - k ln2_hi - k ln2_lo, with ln 2 split into a 32-significant-bit head (k ln2_hi is
//       exact for |k| < 2^21) and its remainder (Cody and Waite's reduction), |r| <= ln(2)/2;
//   e^r = sum_{i <= 13} r^i / i!  (Taylor series, Horner form; truncation below
//       0.3466^14 / 14! = 5e-18 relative);
//   e^x = 2^k e^r, by adding k to the exponent field.
//
// Domain: |x| <= 708 (2^k stays a normal number); x < -708 gives 0, x > 708 gives +inf,
// NaN gives NaN.  Accuracy against the correctly rounded value: a few units in the last
// place of FP64 (tests/test_exp_d_cpu.py).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#ifndef __CUDACC__
#define GPUGA_EXPD_HD inline
#else
#define GPUGA_EXPD_HD __host__ __device__ __forceinline__
#endif

namespace gpuga {

GPUGA_EXPD_HD int64_t expd_bits(double x) {
#ifdef __CUDA_ARCH__
  return __double_as_longlong(x);
#else
  int64_t i;
  std::memcpy(&i, &x, 8);
  return i;
#endif
}

GPUGA_EXPD_HD double expd_from_bits(int64_t i) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double(i);
#else
  double x;
  std::memcpy(&x, &i, 8);
  return x;
#endif
}

// DEG: degree of the Taylor polynomial (13: below an FP64 ulp; 10: truncation below
// 0.3466^11 / 11! = 2.3e-13 relative, three FMAs fewer).
template <int DEG = 13>
GPUGA_EXPD_HD double exp_d(double x) {
  static_assert(DEG >= 8 && DEG <= 13, "exp_d: Taylor degree 8..13");
  const double log2e = 0x1.71547652b82fep+0;      // 1 / ln 2
  const double ln2_hi = 0x1.62e42ff000000p-1;     // ln 2 to 32 significant bits
  const double ln2_lo = -0x1.718432a1b0e26p-35;   // ln 2 - ln2_hi
  const double shifter = 0x1.8p52;                // 1.5 * 2^52
  const double xc = fmin(fmax(x, -708.0), 708.0);
  const double kd_s = fma(xc, log2e, shifter);
  const int64_t k = (int64_t)(int32_t)(uint32_t)expd_bits(kd_s);  // low mantissa bits: k
  const double kd = kd_s - shifter;
  double r = fma(-kd, ln2_hi, xc);
  r = fma(-kd, ln2_lo, r);
  // Taylor coefficients 1/i!, i = DEG .. 0
  constexpr double inv_fact[14] = {1.0,        1.0,         0.5,          1.0 / 6.0,     1.0 / 24.0,
                                   1.0 / 120.0, 1.0 / 720.0, 1.0 / 5040.0, 1.0 / 40320.0, 1.0 / 362880.0,
                                   1.0 / 3628800.0, 1.0 / 39916800.0, 1.0 / 479001600.0, 1.0 / 6227020800.0};
  double p = inv_fact[DEG];
#pragma unroll
  for (int i = DEG - 1; i >= 0; --i) p = fma(p, r, inv_fact[i]);
  const double y = expd_from_bits(expd_bits(p) + (k << 52));
  if (x != x) return x;
  return x < -708.0 ? 0.0 : (x > 708.0 ? INFINITY : y);
}

// The same exponential for arguments the caller knows to be finite: x is clamped to
// [-708, 708] (e^-708 ~ 3e-308 and e^708 ~ 3e307 stand in for 0 and +inf beyond) and a NaN
// argument propagates through the final addition of x - x; no comparisons or selects.
template <int DEG = 13>
GPUGA_EXPD_HD double exp_d_clamped(double x) {
  static_assert(DEG >= 8 && DEG <= 13, "exp_d_clamped: Taylor degree 8..13");
  const double log2e = 0x1.71547652b82fep+0;
  const double ln2_hi = 0x1.62e42ff000000p-1;
  const double ln2_lo = -0x1.718432a1b0e26p-35;
  const double shifter = 0x1.8p52;
  const double xc = fmin(fmax(x, -708.0), 708.0);
  const double kd_s = fma(xc, log2e, shifter);
  const int64_t k = (int64_t)(int32_t)(uint32_t)expd_bits(kd_s);
  const double kd = kd_s - shifter;
  double r = fma(-kd, ln2_hi, xc);
  r = fma(-kd, ln2_lo, r);
  constexpr double inv_fact[14] = {1.0,        1.0,         0.5,          1.0 / 6.0,     1.0 / 24.0,
                                   1.0 / 120.0, 1.0 / 720.0, 1.0 / 5040.0, 1.0 / 40320.0, 1.0 / 362880.0,
                                   1.0 / 3628800.0, 1.0 / 39916800.0, 1.0 / 479001600.0, 1.0 / 6227020800.0};
  double p = inv_fact[DEG];
#pragma unroll
  for (int i = DEG - 1; i >= 0; --i) p = fma(p, r, inv_fact[i]);
  return expd_from_bits(expd_bits(p) + (k << 52)) + (x - x);
}

}  // namespace gpuga
