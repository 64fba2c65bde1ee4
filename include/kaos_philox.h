/*
 * kaos_philox.h -- Philox4x32-10 counter-based generator (Salmon, Moraes,
 * Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11), written
 * from the published round function.  It is the random-number contract of
 * the library: every stochastic kick is a pure function of
 * (seed, particle id, step, stream), so runs are reproducible and a CPU
 * checker that includes this header draws the same uniforms.
 *
 * The reference draws from gfortran's unseeded random_number
 * (_3_1_GaussianRNG.f90:31-33, _3_2_PoissonRNG.f90:35), which cannot be
 * reproduced; only the distributions are kept.
 */
#ifndef KAOS_PHILOX_H
#define KAOS_PHILOX_H

#include <stdint.h>

#if defined(__CUDACC__)
#define KAOS_HD __host__ __device__ __forceinline__
#else
#define KAOS_HD static inline
#endif

#define KAOS_PHILOX_M0 0xD2511F53u
#define KAOS_PHILOX_M1 0xCD9E8D57u
#define KAOS_PHILOX_W0 0x9E3779B9u
#define KAOS_PHILOX_W1 0xBB67AE85u

/* random streams (the fourth counter word, high byte) */
#define KAOS_RNG_HEAT 1u   /* wave-heating Gaussians, per particle/step  */
#define KAOS_RNG_INJECT 2u /* boundary-injection Maxwellian, per particle */
#define KAOS_RNG_NEUT 3u   /* neutral velocity sample, per cell/master    */
#define KAOS_RNG_POIS 4u   /* Poisson collision count, per cell/master    */
#define KAOS_RNG_INIT 5u   /* initial ions (position, population, V)      */

typedef struct {
  uint32_t v[4];
} kaos_u32x4;

KAOS_HD void kaos_mulhilo(uint32_t a, uint32_t b, uint32_t *hi, uint32_t *lo) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  *lo = (uint32_t)p;
}

KAOS_HD kaos_u32x4 kaos_philox(uint32_t c0, uint32_t c1, uint32_t c2,
                               uint32_t c3, uint64_t key) {
  uint32_t k0 = (uint32_t)key, k1 = (uint32_t)(key >> 32);
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    kaos_mulhilo(KAOS_PHILOX_M0, c0, &hi0, &lo0);
    kaos_mulhilo(KAOS_PHILOX_M1, c2, &hi1, &lo1);
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += KAOS_PHILOX_W0;
    k1 += KAOS_PHILOX_W1;
  }
  kaos_u32x4 o;
  o.v[0] = c0;
  o.v[1] = c1;
  o.v[2] = c2;
  o.v[3] = c3;
  return o;
}

/* 53-bit uniform in the open interval (0, 1) from two 32-bit words. */
KAOS_HD double kaos_u01(uint32_t hi, uint32_t lo) {
  uint64_t m = (((uint64_t)hi << 32) | lo) >> 11;
  return ((double)m + 0.5) * 1.1102230246251565404236316680908203125e-16;
}

/* 24-bit uniform in (0, 1) as float, for the mixed-precision kernels. */
KAOS_HD float kaos_u01f(uint32_t w) {
  return ((float)(w >> 8) + 0.5f) * 5.9604644775390625e-08f;
}

#endif
