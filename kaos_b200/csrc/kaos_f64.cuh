// FP64 logarithm, base-2 exponential and sine/cosine of 2 pi u by table
// reduction, for the heating kick of the mixed push in precision mode
// KAOS_PREC_MIXED_K64 (the FP64 path's kick, _8_1_1_0_WaveHeating.f90:
// 141-150, to FP64 accuracy at a fraction of the cost of the general FP64
// library functions).
//
// Method (table-driven reduction, as in Tang's table-driven logarithm and
// exponential, ACM TOMS 15(2) 1989 and 16(4) 1990, here with one 129-entry
// table of 2^(i/128) serving both):
//   log:  x = 2^e m, m in [1, 2); j = nearest integer to 128 log2(m) from an
//         FP32 estimate; z = m 2^(-j/128) lies within 2^(+-(1/256 + 1e-6))
//         of 1, and log(z) = log1p(t), t = z - 1 (|t| < 2.8e-3), is summed
//         to t^6 (the next term is below 2e-19);
//         log x = (128 e + j) ln2/128 + log1p(t).
//   exp2: n = nearest integer to 128 E, f = E - n/128 (|f| <= 1/256);
//         2^E = 2^(n >> 7) 2^((n & 127)/128) e^(f ln2), the last summed to
//         the fifth power (next term below 6e-19).
//   sincos(2 pi u), u in [0, 1]: n = nearest integer to 128 u,
//         x = 2 pi (u - n/128) (|x| <= 0.0246), angle addition with the
//         table's cos, sin of 2 pi n/128 and the Taylor sums of sin x (to
//         x^7) and cos x - 1 (to x^8).
// The tables are built by the caller from the correctly rounded values
// (exp2, sincospi on the device; the C library on the host).
// Errors (tests/test_f64math.py, the host build against long double): the
// logarithms within 2^-51 absolute (relative for results beyond 1 in
// magnitude and next to 1, where the table point is 0; elsewhere the table
// entry's rounding sets an absolute floor, which is what matters when the
// logarithm becomes an exponent or the Box-Muller radius), 2^E and sine,
// cosine within 2^-51 relative and absolute.
#pragma once
#include <math.h>
#include <stdint.h>
#include <string.h>

#ifdef __CUDACC__
#define KF_HD __host__ __device__ __forceinline__
#else
#define KF_HD static inline
#endif

namespace kaos {

constexpr int KF_N = 128;  // table points per octave / per turn

constexpr double KF_LN2 = 0.69314718055994530942;
constexpr double KF_LOG2E = 1.4426950408889634074;
constexpr double KF_TWO_PI = 6.283185307179586477;

KF_HD uint64_t kf_bits(double x) {
#ifdef __CUDA_ARCH__
  return (uint64_t)__double_as_longlong(x);
#else
  uint64_t b;
  memcpy(&b, &x, sizeof b);
  return b;
#endif
}
KF_HD double kf_from_bits(uint64_t b) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)b);
#else
  double x;
  memcpy(&x, &b, sizeof x);
  return x;
#endif
}
// 2^q for -1022 <= q <= 1023
KF_HD double kf_pow2i(int q) { return kf_from_bits((uint64_t)(q + 1023) << 52); }

// FP32 estimate of log2(m), m in [1, 2): picks the table point only
KF_HD float kf_log2_seed(float m) {
#ifdef __CUDA_ARCH__
  float r;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(m));
  return r;
#else
  return log2f(m);
#endif
}

// Reduction of a positive normal x: x = 2^(n/128) (1 + t), returns t and n.
KF_HD double kf_log_reduce(const double *p2, double x, int &n) {
  const uint64_t b = kf_bits(x);
  const int e = (int)(b >> 52) - 1023;
  const double m = kf_from_bits((b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);
  const int j = (int)rintf(128.0f * kf_log2_seed((float)m));  // 0 .. 128
  n = 128 * e + j;
  // m 2^(-j/128) = m 2^((128 - j)/128) / 2 (one rounding)
  return fma(m, 0.5 * p2[KF_N - j], -1.0);
}
// log1p(t) for |t| < 2.8e-3
KF_HD double kf_log1p_small(double t) {
  const double p = fma(t, fma(t, fma(t, fma(t, fma(t, -1.0 / 6.0, 0.2), -0.25), 1.0 / 3.0),
                              -0.5), 1.0);
  return t * p;
}

// Natural logarithm of a positive normal x.
KF_HD double kf_ln(const double *p2, double x) {
  int n;
  const double t = kf_log_reduce(p2, x, n);
  return fma((double)n, KF_LN2 / 128.0, kf_log1p_small(t));
}
// Base-2 logarithm of a positive normal x.
KF_HD double kf_log2(const double *p2, double x) {
  int n;
  const double t = kf_log_reduce(p2, x, n);
  return fma(kf_log1p_small(t), KF_LOG2E, (double)n * (1.0 / 128.0));
}

// 2^E for -1000 < E < 1000.
KF_HD double kf_exp2(const double *p2, double E) {
  const double nd = rint(E * 128.0);
  const int n = (int)nd;
  const double g = fma(nd, -1.0 / 128.0, E) * KF_LN2;  // |g| <= 2.71e-3
  // e^g - 1 to g^5
  const double em1 =
      g * fma(g, fma(g, fma(g, fma(g, 1.0 / 120.0, 1.0 / 24.0), 1.0 / 6.0), 0.5), 1.0);
  const double t = p2[n & (KF_N - 1)];
  return fma(t, em1, t) * kf_pow2i(n >> 7);
}

// cos and sin of 2 pi u for u in [0, 1]; cs holds (cos, sin) of 2 pi i/128
// as pairs, i = 0 .. 128.
KF_HD void kf_sincos2pi(const double *cs, double u, double &s, double &c) {
  const double nd = rint(u * 128.0);
  const int n = (int)nd;
  const double x = fma(nd, -1.0 / 128.0, u) * KF_TWO_PI;
  const double x2 = x * x;
  const double sx = x * fma(x2, fma(x2, fma(x2, -1.0 / 5040.0, 1.0 / 120.0), -1.0 / 6.0), 1.0);
  const double cm1 =
      x2 * fma(x2, fma(x2, fma(x2, 1.0 / 40320.0, -1.0 / 720.0), 1.0 / 24.0), -0.5);
  const double C = cs[2 * n], S = cs[2 * n + 1];
  c = C + fma(C, cm1, -S * sx);
  s = S + fma(S, cm1, C * sx);
}

}  // namespace kaos
