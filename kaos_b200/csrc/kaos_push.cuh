// kaos_push.cuh -- the fused per-particle step: KineticUpdateA/B/C forces,
// modified RK4 (k3 = k2), wave heating, start-of-step binning and the
// per-step re-projection onto the flux tube (RK4DipolePolynomialSolver),
// one thread per particle with every RK stage in registers.
//
// Reference: KineticRK4UpdateSub _8_1_KineticRK4Update.f90:29-315,
// KineticUpdateASub _8_1_1_KineticUpdateA.f90:117-1392,
// KineticUpdateBSub _8_1_2_KineticUpdateB.f90:31-786,
// KineticUpdateCSub _8_1_3_KineticUpdateC.f90:31-809,
// RK4DipolePolynomialSolverSub _8_1_4_RK4DipolePolynomialSolver.f90:26-134,
// WaveHeatingSub _8_1_1_0_WaveHeating.f90:32-312.
#pragma once
#include "kaos_common.cuh"
#include "kaos_f64.cuh"

namespace kaos {

__constant__ VGridC c_vg;

struct PushArgs {
  const TubeD *tubes;
  const int *blk_tube;       // work item -> tube
  const int64_t *blk_start;  // work item -> first ion (tube-relative)
  int nitems;                // work items (tube, chunk of ions)
  int chunk;                 // ions per work item
  int nqs;                   // cells per tube in the shared-memory layout
  const int64_t *nlive;
  Ions ion;
  CellTables ct;
  Accum acc;
  double h, ms, qs;
  uint64_t seed;
  uint32_t step;
  ForceFlags ff;
  int icr, icrcoh;
  int bin;        // accumulate start-of-step counts (master step)
  int prologue;   // re-interpolate the cached fields at qk4 first
  int write_qind; // store Qindk1 (needed by the next boundary/collision pass)
  int write_qk4;  // store q at the k4 point (next step is a master step)
  int exporting;  // also fill the full phase-space histogram
  int bin_only;   // count only, do not advance (first step statistics)
  uint32_t *status;
  // charge exchange on: per (selection chunk, cell) counts of the Qindk1
  // written by this push, for the next step's in-order selection
  unsigned *cxc;
  const int *tube_cx0;
  int cx_stride, cx_chunk;
  // graph replay: the step number is read from device memory
  const uint32_t *dstep;
  // Philox key schedule of the seed: key words of round r at rk[2r], rk[2r+1]
  uint32_t rk[20];
};

// Flush a block's per-cell Qindk1 counts into its selection-chunk row.
__device__ __forceinline__ void flush_cx_counts(const PushArgs &a, int t,
                                                int64_t beg, int nq,
                                                const unsigned *HC) {
  __syncthreads();
  unsigned *row = a.cxc + (int64_t)(a.tube_cx0[t] + (int)(beg / a.cx_chunk)) * a.cx_stride;
  for (int k = threadIdx.x; k < nq; k += blockDim.x)
    if (HC[k]) atomicAdd(row + k, HC[k]);
}

// ---- warp-aggregated counter increment -----------------------------------
__device__ __forceinline__ void agg_inc(unsigned int *base, int64_t idx) {
  unsigned mask = __activemask();
  unsigned peers = __match_any_sync(mask, (unsigned long long)idx);
  int leader = __ffs(peers) - 1;
  if ((int)(threadIdx.x & 31) == leader)
    atomicAdd(base + idx, (unsigned)__popc(peers));
}

// Start-of-step binning of one ion (IonParticleCountsSub counts by
// Qindk1/V*indk1, _8_3_1_IonParticleCounts.f90:63-80, :336-357, :612-632).
// Only per-cell counts and the per-axis marginals are kept: every moment
// integrand of _8_6_1.._8_6_6 is a sum of single-axis terms.
__device__ __forceinline__ void hist_inc(const Accum &acc, const TubeD &T,
                                         int qi, int b1, int b2, int bp) {
  const bool d3 = c_vg.three_d;
  int64_t nv = d3 ? (int64_t)c_vg.n1 * c_vg.n2 * c_vg.npar
                  : (int64_t)c_vg.n1 * c_vg.npar;
  int64_t b = d3 ? ((int64_t)b1 * c_vg.n2 + b2) * c_vg.npar + bp
                 : (int64_t)b1 * c_vg.npar + bp;
  atomicAdd(acc.hist + T.hoff + (int64_t)qi * nv + b, 1u);
}

__device__ __forceinline__ void accumulate(const Accum &acc, const TubeD &T,
                                           int qi, int b1, int b2, int bp,
                                           int exporting) {
  if (qi < 0) return;
  const int64_t gc = T.coff + qi;
  agg_inc(acc.cnt, gc);
  const bool d3 = c_vg.three_d;
  if (b1 < 0 || bp < 0 || (d3 && b2 < 0)) return;
  atomicAdd(acc.mpar + gc * c_vg.npar + bp, 1u);
  atomicAdd(acc.m1 + gc * c_vg.n1 + b1, 1u);
  if (d3) atomicAdd(acc.m2 + gc * c_vg.n2 + b2, 1u);
  if (exporting) hist_inc(acc, T, qi, b1, b2, bp);
}

// Block-private binning window: the counters of BIN_WIN consecutive cells
// starting at the cell of the block's first ion live in shared memory (the
// ion arrays stay nearly ordered by cell: ions are created cell by cell and
// move a small fraction of a cell per step); ions outside the window go to
// the global counters.  The window is flushed once per block.
constexpr int BIN_WIN = 4;

__device__ __forceinline__ int bin_win_size() {
  return BIN_WIN * (1 + c_vg.npar + c_vg.n1 + (c_vg.three_d ? c_vg.n2 : 0));
}

struct BinWin {
  int lo;
  unsigned *s;  // [cnt BIN_WIN][mpar BIN_WIN*npar][m1 BIN_WIN*n1][m2 BIN_WIN*n2]
};

__device__ __forceinline__ BinWin bin_win_init(unsigned *base, int first_cell,
                                               int nq) {
  BinWin W;
  W.lo = max(0, min(first_cell - 1, nq - BIN_WIN));
  W.s = base;
  const int n = bin_win_size();
  for (int k = threadIdx.x; k < n; k += blockDim.x) base[k] = 0u;
  return W;  // the caller synchronises before the first use
}

__device__ __forceinline__ void accumulate_win(const Accum &acc, const TubeD &T,
                                               const BinWin &W, int qi, int b1,
                                               int b2, int bp, int exporting) {
  if (qi < 0) return;
  const int wc = qi - W.lo;
  if ((unsigned)wc >= (unsigned)BIN_WIN) {
    accumulate(acc, T, qi, b1, b2, bp, exporting);
    return;
  }
  // the cell count: one shared-memory atomic per distinct cell among the
  // warp's ions (they mostly share one) instead of one per ion
  const unsigned peers = __match_any_sync(__activemask(), wc);
  if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(W.s + wc, (unsigned)__popc(peers));
  const bool d3 = c_vg.three_d;
  if (b1 < 0 || bp < 0 || (d3 && b2 < 0)) return;
  unsigned *mp = W.s + BIN_WIN, *m1 = mp + BIN_WIN * c_vg.npar,
           *m2 = m1 + BIN_WIN * c_vg.n1;
  atomicAdd(mp + wc * c_vg.npar + bp, 1u);
  atomicAdd(m1 + wc * c_vg.n1 + b1, 1u);
  if (d3) atomicAdd(m2 + wc * c_vg.n2 + b2, 1u);
  if (exporting) hist_inc(acc, T, qi, b1, b2, bp);
}

__device__ __forceinline__ void bin_win_flush(const Accum &acc, const TubeD &T,
                                              const BinWin &W) {
  __syncthreads();
  const int np = c_vg.npar, n1 = c_vg.n1, n2 = c_vg.three_d ? c_vg.n2 : 0;
  const int n = bin_win_size();
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const unsigned v = W.s[k];
    if (!v) continue;
    int r = k, wc, b;
    unsigned *dst;
    if (r < BIN_WIN) {
      wc = r;
      dst = acc.cnt + (T.coff + W.lo + wc);
    } else if ((r -= BIN_WIN) < BIN_WIN * np) {
      wc = r / np; b = r - wc * np;
      dst = acc.mpar + (int64_t)(T.coff + W.lo + wc) * np + b;
    } else if ((r -= BIN_WIN * np) < BIN_WIN * n1) {
      wc = r / n1; b = r - wc * n1;
      dst = acc.m1 + (int64_t)(T.coff + W.lo + wc) * n1 + b;
    } else {
      r -= BIN_WIN * n1;
      wc = r / n2; b = r - wc * n2;
      dst = acc.m2 + (int64_t)(T.coff + W.lo + wc) * n2 + b;
    }
    atomicAdd(dst, v);
  }
}

// Field magnitude at q by linear interpolation between cell centres with
// constant half cells at both ends (_8_7_AmbipolarEfield.f90:1453-2722).
// centre_segment gives the segment of s = sgn*q: 0 below the first centre,
// nq above the last, else the smallest k in [1, nq-1] with s <= C[k] (the
// same k as a bisection), found by walking from the ion's cell since q_k4
// lies within a cell or two of it; -1 outside the grid (the ion keeps its
// field values).
__device__ __forceinline__ int centre_segment(const double *E, const double *C,
                                              int nq, double s, int guess) {
  if (s < E[0] || s > E[nq]) return -1;
  if (s <= C[0]) return 0;
  if (s >= C[nq - 1]) return nq;
  int k = min(max(guess, 1), nq - 1);
  while (k > 1 && s <= C[k - 1]) --k;
  while (k < nq - 1 && s > C[k]) ++k;
  return k;
}

// y1 + ((q - x1) / (x2 - x1)) (y2 - y1) (LinInterpsub, _KineticMainParams
// .f90:810-815) on segment k; frac = (q - x1) / (x2 - x1) is shared by the
// fields interpolated at the same q.
__device__ __forceinline__ double interp_frac(int k, const double *qC, int nq,
                                              double q) {
  if (k == 0 || k == nq) return 0.0;
  const double x1 = qC[k - 1], x2 = qC[k];
  return (q - x1) / (x2 - x1);
}

__device__ __forceinline__ double interp_at(int k, const double *Eg, int nq,
                                            double frac) {
  if (k == 0) return Eg[0];
  if (k == nq) return Eg[nq - 1];
  return Eg[k - 1] + (frac * (Eg[k] - Eg[k - 1]));
}

__device__ __forceinline__ void field_prologue(const PushArgs &a,
                                               const TubeD &T, const double *E,
                                               const double *C, double qk,
                                               int guess, double &aea,
                                               double &ag) {
  const int k = centre_segment(E, C, T.nq, T.sgn * qk, guess);
  if (k < 0) return;
  const double qm = T.qs / T.ms;
  const double frac = interp_frac(k, a.ct.qGC + T.coff, T.nq, qk);
  if (a.ff.eamb) {
    const double v = interp_at(k, a.ct.EAmag + T.coff, T.nq, frac);
    double e = a.ff.eambsign ? v : fabs(v);
    aea = (e == 0.0) ? 0.0 : (a.ff.eambsign ? qm * e : fabs(qm * e));
  }
  if (a.ff.grav) {
    const double v = interp_at(k, a.ct.EG + T.coff, T.nq, frac);
    double e = fabs(v);
    ag = (e == 0.0) ? 0.0 : fabs(qm * e);
  }
}

// Two Box-Muller Gaussians (cos and sin branches) from one Philox draw
// keyed by (seed, particle id, step): GaussianRNGSub's transform
// (_3_1_GaussianRNG.f90:33) with both outputs used.
__device__ __forceinline__ void gauss2_64(uint64_t seed, uint64_t id,
                                          uint32_t step, uint32_t stream,
                                          double &g1, double &g2) {
  kaos_u32x4 w = kaos_philox((uint32_t)id, (uint32_t)(id >> 32), step,
                             stream << 24, seed);
  double u1 = kaos_u01(w.v[0], w.v[1]);
  double u2 = kaos_u01(w.v[2], w.v[3]);
  double R = sqrt(-2.0 * log(u1)), sn, cs;
  sincospi(2.0 * u2, &sn, &cs);
  g1 = R * cs;
  g2 = R * sn;
}
__device__ __forceinline__ void gauss2_32(uint64_t seed, uint64_t id,
                                          uint32_t step, uint32_t stream,
                                          float &g1, float &g2) {
  kaos_u32x4 w = kaos_philox((uint32_t)id, (uint32_t)(id >> 32), step,
                             stream << 24, seed);
  float u1 = kaos_u01f(w.v[0]), u2 = kaos_u01f(w.v[2]);
  float R = sqrtf(fmaxf(-2.0f * __logf(u1), 0.0f)), sn, cs;
  __sincosf(6.2831853071795865f * u2, &sn, &cs);
  g1 = R * cs;
  g2 = R * sn;
}
// Single Gaussian (injection): cos branch of one draw.
__device__ __forceinline__ double gauss64(uint64_t seed, uint64_t id,
                                          uint32_t step, uint32_t stream,
                                          uint32_t sub) {
  kaos_u32x4 w = kaos_philox((uint32_t)id, (uint32_t)(id >> 32), step,
                             (stream << 24) | sub, seed);
  double u1 = kaos_u01(w.v[0], w.v[1]);
  double u2 = kaos_u01(w.v[2], w.v[3]);
  return sqrt(-2.0 * log(u1)) * cos(2.0 * PI * u2);
}

// Per-cell wave-heating constants, precomputed on the host from the ICR
// tables (_1_SimParameterization.f90:1408-1444):
//   K_i = h sqrt(q^2 xi_i eta S0 / (2 m^2 pi)),  c_i = chi_i / 2,
//   w0 = 1/OmegaG0, lam = lambdaPerp.
template <typename T> struct HeatC {
  T K1, K2, c1, c2, iom0, lam;
};

// WaveHeatingSub kicks (_8_1_1_0_WaveHeating.f90:72-312).  With
// D_i = q^2/(2m^2) xi_i eta S0 (Omega/Omega0)^-chi_i Sigma^-3,
// eps = |V|/(Omega sum ds), tau = 1/((Omega/2pi) sqrt eps) and the kick
// (h/tau) sqrt(2 D_i tau) G_i, the algebra reduces to
//   kick_i = K_i x^(-chi_i/2) Sigma^(-3/2) sqrt(Omega s) G_i,  s = sqrt(eps),
// applied while h <= tau, i.e. h Omega s <= 2 pi (stochastic branch);
// the coherent branch kicks |Vperp| by sqrt(k1^2+k2^2) G1 with a uniform
// gyro-angle.  invOm = 1/Omega is passed in (no division needed).
template <typename T>
__device__ __forceinline__ void heat(const PushArgs &a, uint32_t step,
                                     const HeatC<T> &c, uint64_t id,
                                     T invsumds, T Om, T invOm, T vparabs,
                                     T &v1, T &v2) {
  const bool f64 = sizeof(T) == 8;
  const T x = Om * c.iom0;
  T e1, e2;
  if (f64) {
    double lx = log((double)x);
    e1 = (T)exp(-(double)c.c1 * lx);
    e2 = (c.c2 == c.c1) ? e1 : (T)exp(-(double)c.c2 * lx);
  } else {
    float lx = __logf((float)x);
    e1 = (T)__expf(-(float)c.c1 * lx);
    e2 = (c.c2 == c.c1) ? e1 : (T)__expf(-(float)c.c2 * lx);
  }
  const T s = sqrt(vparabs * invsumds * invOm);
  const T w = sqrt(Om * s);
  T k1 = c.K1 * e1 * w, k2 = c.K2 * e2 * w;
  if (c.lam != T(0)) {
    const T vpm = sqrt(v1 * v1 + v2 * v2);
    const T Sig = T(2.0 * PI) * vpm * invOm / c.lam;
    if (Sig >= T(1)) {
      const T f = T(1) / (Sig * sqrt(Sig));
      k1 *= f;
      k2 *= f;
    }
  }
  T G1, G2;
  if (f64) {
    double g1, g2;
    gauss2_64(a.seed, id, step, KAOS_RNG_HEAT, g1, g2);
    G1 = (T)g1;
    G2 = (T)g2;
  } else {
    float g1, g2;
    gauss2_32(a.seed, id, step, KAOS_RNG_HEAT, g1, g2);
    G1 = (T)g1;
    G2 = (T)g2;
  }
  if (a.icrcoh) {
    const T vpn = fabs(sqrt(v1 * v1 + v2 * v2) + sqrt(k1 * k1 + k2 * k2) * G1);
    kaos_u32x4 r = kaos_philox((uint32_t)id, (uint32_t)(id >> 32), step,
                               (KAOS_RNG_HEAT << 24) | 2u, a.seed);
    const T ga = (T)kaos_u01(r.v[0], r.v[1]) * T(2.0 * PI);
    v1 = vpn * cos(ga);
    v2 = vpn * sin(ga);
    return;
  }
  if (a.h * (double)(Om * s) <= 2.0 * PI) {
    v1 = v1 + k1 * G1;
    v2 = v2 + k2 * G2;
  }
}

// Philox4x32-10 (include/kaos_philox.h) with the key schedule, the same for
// every particle, read from the kernel arguments (rk: key words of round r
// at rk[2r], rk[2r+1]): the same output words.
__device__ __forceinline__ kaos_u32x4 philox_rk(const uint32_t (&rk)[20], uint32_t c0,
                                                uint32_t c1, uint32_t c2,
                                                uint32_t c3) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)KAOS_PHILOX_M0 * c0;
    const uint64_t p1 = (uint64_t)KAOS_PHILOX_M1 * c2;
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ rk[2 * r];
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ rk[2 * r + 1];
    c1 = (uint32_t)p1;
    c3 = (uint32_t)p0;
    c0 = n0;
    c2 = n2;
  }
  kaos_u32x4 o;
  o.v[0] = c0;
  o.v[1] = c1;
  o.v[2] = c2;
  o.v[3] = c3;
  return o;
}

// Uniform in (0, 1) from the high 23 bits of w, (2 (w >> 9) + 1) 2^-24, made
// from the mantissa bits of a float in [1, 2) (exact; within 2^-25 of
// kaos_u01f(w)).
__device__ __forceinline__ float u01_bits(uint32_t w) {
  return __uint_as_float(0x3f800000u | (w >> 9)) - 0x1.fffffep-1f;
}

// Single MUFU operations of the mixed push, denormals flushed: reciprocal,
// sine and cosine (radians).
__device__ __forceinline__ float rcpa(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float sina(float x) {
  float r;
  asm("sin.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float cosa(float x) {
  float r;
  asm("cos.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// field_prologue for the mixed push, where q_k4 is held in FP32: the same
// segment (walk over the oriented cell centres C = sgn qGC in shared
// memory), the fraction with a one-instruction reciprocal, and the
// interpolation and q/m scaling in FP32 from the cell fields FE (EAmag, EG
// per cell, in shared memory).
__device__ __forceinline__ void field_prologue32(const ForceFlags &ff,
                                                 const TubeD &T, const double *E,
                                                 const double *C, const float2 *FE,
                                                 float qk, int guess, float qm,
                                                 float &aea, float &ag) {
  const int nq = T.nq;
  const int k = centre_segment(E, C, nq, T.sgn * (double)qk, guess);
  if (k < 0) return;
  float2 f;
  if (k == 0) {
    f = FE[0];
  } else if (k == nq) {
    f = FE[nq - 1];
  } else {
    const double x1 = T.sgn * C[k - 1], x2 = T.sgn * C[k];
    const float frac = (float)((double)qk - x1) * rcpa((float)(x2 - x1));
    const float2 y1 = FE[k - 1], y2 = FE[k];
    f.x = fmaf(frac, y2.x - y1.x, y1.x);
    f.y = fmaf(frac, y2.y - y1.y, y1.y);
  }
  if (ff.eamb) {
    const float e = ff.eambsign ? f.x : fabsf(f.x);
    aea = (e == 0.0f) ? 0.0f : (ff.eambsign ? qm * e : fabsf(qm * e));
  }
  if (ff.grav) {
    const float e = fabsf(f.y);
    ag = (e == 0.0f) ? 0.0f : fabsf(qm * e);
  }
}

// Velocity-bin search of the mixed push from a lookup table: VTAB uniform
// slots over the axis hold the bin of each slot's left end, and a short walk
// over the FP64 edges finishes the search.
// The walk establishes both edge conditions of vbin (v <= e[b+1], and
// v > e[b] unless b = 0) in FP64, so the result equals vbin's on the FP64
// edges whatever the table holds.
constexpr int VTAB = 256;
struct VBinTab {
  double e0, iw;             // first edge, VTAB / (last edge - first edge)
  unsigned char t[VTAB];     // bin at each slot's left end (n <= 128)
};
// Dynamic shared memory of the mixed push's bin searches: alignment slack,
// three FP64 edge arrays and three lookup tables.
constexpr size_t BINS_SMEM_BYTES = 16 + 3 * (MAXV + 1) * sizeof(double) + 3 * sizeof(VBinTab);

// All threads of the block; edges e[0..n] in shared memory already visible,
// and the caller synchronises before the table is used.
__device__ __forceinline__ void build_vbin_tab(VBinTab &T, const double *e, int n) {
  if (threadIdx.x == 0) {
    T.e0 = e[0];
    T.iw = (double)VTAB / (e[n] - e[0]);
  }
  for (int k = threadIdx.x; k < VTAB; k += blockDim.x) {
    const double v = e[0] + (e[n] - e[0]) * ((double)k / (double)VTAB);
    T.t[k] = (unsigned char)max(vbin(e, n, v), 0);
  }
}

__device__ __forceinline__ int vbin_tab(const VBinTab &T, const double *e, int n,
                                        double v) {
  if (!(v >= e[0] && v <= e[n])) return -1;
  // slot floor((v - e0) iw): round-to-nearest of (v - e0) iw - 1/2 read from
  // the low word of its sum with 1.5 * 2^52 (no conversion instruction)
  const double sl = fma(v - T.e0, T.iw, -0.5) + 6755399441055744.0;
  const int s = min(max((int)__double2loint(sl), 0), VTAB - 1);
  int b = T.t[s];
  // one predicated step up settles almost every value (the table gives the
  // bin of the slot's left end); the loops finish the rare rest exactly
  b += (b < n - 1 && v > e[b + 1]) ? 1 : 0;
  if (__builtin_expect((b > 0 && v <= e[b]) || (b < n - 1 && v > e[b + 1]), 0)) {
    while (b > 0 && v <= e[b]) --b;
    while (b < n - 1 && v > e[b + 1]) ++b;
  }
  return b;
}

// Hardware base-2 logarithm and exponential (MUFU, flush-to-zero).
__device__ __forceinline__ float lg2f(float x) {
  float r;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float ex2f(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// The Gaussian pair of the mixed push's heating kick: Box-Muller
// (GaussianRNGSub's transform, _3_1_GaussianRNG.f90:33, both branches) in
// FP32 from the high 23 bits of Philox words 0 and 2 of the draw keyed by
// (seed, particle id, step, heating stream), with the hardware logarithm,
// reciprocal square root, sine and cosine.  Also evaluated by the
// diagnostic sampler kaos_sample_rng.
__device__ __forceinline__ void gauss2_mix(const uint32_t (&rk)[20], uint64_t id,
                                           uint32_t step, float &g1, float &g2) {
  const kaos_u32x4 w = philox_rk(rk, (uint32_t)id, (uint32_t)(id >> 32), step,
                                 KAOS_RNG_HEAT << 24);
  const float u1 = u01_bits(w.v[0]), u2 = u01_bits(w.v[2]);
  // -2 ln u1 > 0; the hardware logarithm's absolute error (~2^-22) can give
  // a tiny negative value for u1 just below 1
  const float t = fmaxf(-1.38629436f * lg2f(u1), 1e-30f);
  const float R = t * rsq(t);
  const float ang = 6.2831853f * u2;
  g1 = R * cosa(ang);
  g2 = R * sina(ang);
}

// The stochastic WaveHeatingSub kick in the mixed push, in log form: the
// product K_i x^(-c_i) (Om s)^(1/2) of heat() is one base-2 exponential,
//   kick_i = K_i G_i 2^(-c_i log2(Om/Om0) + log2(Om |V||| / sum ds)/4 - pen),
// the branch test h Om s <= 2 pi becomes Om |V||| / sum ds <= (2 pi/h)^2 and
// Sigma^(-3/2) for lambda != 0 becomes pen = 1.5 log2 Sigma when Sigma >= 1,
// log2 Sigma = log2(Vperp^2)/2 + log2(2 pi/lambda) - log2 Om.
// The Gaussians are the same Box-Muller pair of one Philox draw as
// gauss2_32.  hk (8 per cell): K1 K2 c1 c2 log2(1/Om0) lambda
// log2(2 pi/lambda) 0.  The kicks come back in dv1, dv2 (zero outside the
// stochastic regime); the caller adds them to its FP64 Vperp.
__device__ __forceinline__ void heat32(const PushArgs &a, uint32_t step,
                                       const float *hk, uint64_t id,
                                       float invsumds, float ylim, float Om,
                                       float vabs, float vp2, float &dv1,
                                       float &dv2) {
  dv1 = dv2 = 0.0f;
  const float y = Om * vabs * invsumds;  // (Om s)^2
  if (!(y <= ylim)) return;
  const float4 h0 = *(const float4 *)hk, h1 = *(const float4 *)(hk + 4);
  const float LOm = lg2f(Om);
  float b = 0.25f * lg2f(y);
  if (h1.y != 0.0f) {  // lambda != 0
    const float ls = fmaf(0.5f, lg2f(vp2), h1.z) - LOm;
    if (ls >= 0.0f) b -= 1.5f * ls;
  }
  const float lx = LOm + h1.x;
  const float e1 = ex2f(fmaf(-h0.z, lx, b));
  const float e2 = (h0.w == h0.z) ? e1 : ex2f(fmaf(-h0.w, lx, b));
  float G1, G2;
  gauss2_mix(a.rk, id, step, G1, G2);
  dv1 = h0.x * e1 * G1;
  dv2 = h0.y * e2 * G2;
}

// The tables of kaos_f64.cuh in shared memory (allocated only in the
// kernels that call this): 2^(i/128), i = 0..128, then the (cos, sin) pairs
// of 2 pi i/128.  Filled by kf_tables_fill before the block's first barrier.
__device__ __forceinline__ double *kf_tables() {
  __shared__ double t[3 * (KF_N + 1)];
  return t;
}
__device__ __forceinline__ void kf_tables_fill(double *t) {
  for (int i = threadIdx.x; i <= KF_N; i += blockDim.x) {
    double sn, cs;
    t[i] = exp2((double)i / KF_N);
    sincospi((double)i / (KF_N / 2), &sn, &cs);
    t[KF_N + 1 + 2 * i] = cs;
    t[KF_N + 2 + 2 * i] = sn;
  }
}

// gauss2_64's Gaussian pair (the same Philox words, 53-bit uniforms) through
// the table-reduced logarithm and sine/cosine; kt = kf_tables().  Also
// evaluated by the diagnostic sampler kaos_sample_rng.
__device__ __forceinline__ void gauss2_64t(const uint32_t (&rk)[20], const double *kt,
                                           uint64_t id, uint32_t step, double &g1,
                                           double &g2) {
  const kaos_u32x4 w = philox_rk(rk, (uint32_t)id, (uint32_t)(id >> 32), step,
                                 KAOS_RNG_HEAT << 24);
  const double R = sqrt(-2.0 * kf_ln(kt, kaos_u01(w.v[0], w.v[1])));
  double sn, cn;
  kf_sincos2pi(kt + KF_N + 1, kaos_u01(w.v[2], w.v[3]), sn, cn);
  g1 = R * cn;
  g2 = R * sn;
}

// The stochastic WaveHeatingSub kick of heat<double> (the FP64 path's kick)
// for the mixed push in precision mode KAOS_PREC_MIXED_K64, every factor in
// FP64 through the table-reduced functions of kaos_f64.cuh.  In log form,
// as in heat32,
//   kick_i = K_i G_i 2^E_i,  E_i = -c_i log2(Om/Om0) + log2(y Sig^-6)/4,
// y = Om |V||| / sum ds = (Om s)^2, the Sig^-6 factor (Sig = 2 pi Vperp /
// (Om lambda)) only for lambda != 0 and Sig >= 1; applied while
// y <= (2 pi/h)^2 (h Om s <= 2 pi).  The Gaussians are gauss2_64's pair
// from the same Philox words (53-bit uniforms); the kicks agree with
// heat<double>'s to a few units in the last place.  A kick below 1e-75 of
// its scale (y Sig^-6 < 1e-300) is left out: added to an FP64 velocity it
// changes nothing.
__device__ __forceinline__ void heat64t(const PushArgs &a, uint32_t step,
                                        const double *kt, const CellTables &ct,
                                        int64_t g, uint64_t id, double invsumds,
                                        double ylim, double Om, double invOm,
                                        double vabs, double &v1, double &v2) {
  double arg = Om * vabs * invsumds;  // y
  if (!(arg <= ylim)) return;         // beyond the stochastic regime
  const double lam = ct.lambdaPerp[g];
  if (lam != 0.0) {
    const double sk = (2.0 * PI) * invOm / lam;
    const double S2 = sk * sk * fma(v1, v1, v2 * v2);  // Sig^2
    if (S2 >= 1.0) arg = arg / (S2 * S2 * S2);
  }
  if (!(arg > 1e-300)) return;
  double G1, G2;
  gauss2_64t(a.rk, kt, id, step, G1, G2);
  const double *p2 = kt;
  const double c1 = ct.hc1[g], c2 = ct.hc2[g];
  const double lx = kf_log2(p2, Om * ct.hiom0[g]);
  const double b = 0.25 * kf_log2(p2, arg);
  const double e1 = kf_exp2(p2, fma(-c1, lx, b));
  const double e2 = (c2 == c1) ? e1 : kf_exp2(p2, fma(-c2, lx, b));
  v1 = fma(ct.hK1[g] * e1, G1, v1);
  v2 = fma(ct.hK2[g] * e2, G2, v2);
}

// Positive root u = r/RE of q^2 u^4 + u/p - 1 = 0 by Newton from u0 (the
// function is increasing and convex for u > 0: the root is unique).  The
// derivative is inverted in FP32 (correctly rounded); each step still
// contracts the error by ~1e-7 on top of the quadratic term.
__device__ __forceinline__ double quartic_newton(double q, double ip, double u,
                                                 int iters) {
  const double q2 = q * q;
  for (int k = 0; k < iters; ++k) {
    const double u2 = u * u;
    const double f = fma(q2 * u2, u2, fma(u, ip, -1.0));
    const double fp = fma(4.0 * q2 * u2, u, ip);
    const float r = __frcp_rn((float)fp);
    u = fma(-f, (double)r, u);
  }
  return u;
}

// The same root by Newton steps (derivative inverted in FP32, correctly
// rounded) until the correction falls below 1e-15 of u -- the error left is
// then ~1e-22 -- or maxit steps: for guesses of unknown quality (a tube moved
// to a new L-shell, a cell's linear guess).
__device__ __forceinline__ double quartic_newton_conv(double q, double ip, double u,
                                                      int maxit) {
  const double q2 = q * q;
  for (int k = 0; k < maxit; ++k) {
    const double u2 = u * u;
    const double f = fma(q2 * u2, u2, fma(u, ip, -1.0));
    const double fp = fma(4.0 * q2 * u2, u, ip);
    const double du = f * (double)__frcp_rn((float)fp);
    u -= du;
    if (fabs(du) <= 1e-15 * u) break;
  }
  return u;
}

// The same root from a guess within ~1e-4: one Newton step with the
// derivative inverted in FP32, then a chord step reusing that inverse (the
// derivative changes by ~1e-4 between the two points, so the chord step
// contracts the error by that much more; ~1e-17 relative on the benchmark
// tubes' per-cell quadratic guesses, whose error is below 3.2e-5).
__device__ __forceinline__ double quartic_newton_chord(double q, double ip,
                                                       double u) {
  const double q2 = q * q;
  double u2 = u * u;
  double f = fma(q2 * u2, u2, fma(u, ip, -1.0));
  const double r = (double)rcpa((float)fma(4.0 * q2 * u2, u, ip));
  u = fma(-f, r, u);
  u2 = u * u;
  f = fma(q2 * u2, u2, fma(u, ip, -1.0));
  return fma(-f, r, u);
}

// Cell search starting from the cell of the previous step (particles move a
// small fraction of a cell per step); falls back to the bisection.
__device__ __forceinline__ int cell_search_from(const double *E, int nq,
                                                double s, int g) {
  if (g >= 0 && g < nq) {
    if (s <= E[g + 1] && (g == 0 ? s >= E[0] : s > E[g])) return g;
    if (g + 1 < nq && s > E[g + 1] && s <= E[g + 2]) return g + 1;
    if (g > 0 && s <= E[g] && (g == 1 ? s >= E[0] : s > E[g - 1])) return g - 1;
  }
  return cell_search(E, nq, s);
}

// Copy the velocity-cell edges of the three axes into shared memory.
template <typename T>
__device__ __forceinline__ void load_vgrid_smem(const T *e1, const T *e2,
                                                const T *ep, T *s1, T *s2,
                                                T *sp) {
  for (int k = threadIdx.x; k <= MAXV; k += blockDim.x) {
    s1[k] = e1[k];
    s2[k] = e2[k];
    sp[k] = ep[k];
  }
}

// Load this block's tube and its oriented cell edges / centres into smem.
__device__ __forceinline__ void load_tube_smem(const PushArgs &a, int t,
                                               TubeD &T, double *E,
                                               double *Cc) {
  T = a.tubes[t];
  const double *qGL = a.ct.qGL + T.coff, *qGH = a.ct.qGH + T.coff,
               *qGC = a.ct.qGC + T.coff;
  for (int k = threadIdx.x; k <= T.nq; k += blockDim.x) {
    E[k] = (k < T.nq) ? T.sgn * qGL[k] : T.sgn * qGH[T.nq - 1];
    if (k < T.nq) Cc[k] = T.sgn * qGC[k];
  }
}

template <typename T>
__device__ __forceinline__ HeatC<T> heat_consts(const CellTables &c, int64_t g) {
  HeatC<T> h;
  h.K1 = (T)c.hK1[g];
  h.K2 = (T)c.hK2[g];
  h.c1 = (T)c.hc1[g];
  h.c2 = (T)c.hc2[g];
  h.iom0 = (T)c.hiom0[g];
  h.lam = (T)c.lambdaPerp[g];
  return h;
}

// ---------------------------------------------------------------------------
// FP64 kernel: ions stored as meridian-plane (rho, z) in FP64.
template <bool THREE_D, bool PERSIST>
__global__ void __launch_bounds__(256, 2) k_push64(PushArgs a) {
  extern __shared__ double sm[];
  const int nqmax = a.nqs;
  double *E = sm, *Cc = sm + nqmax + 1;
  unsigned *HC = (unsigned *)(Cc + nqmax);
  const double h = a.h, hh = 0.5 * a.h, h6 = a.h / 6.0, hsq2 = 0.5 * a.h * a.h;
  const uint32_t step = a.dstep ? *a.dstep : a.step;
  Ions I = a.ion;
  TubeD T;
  int tcur = -1;
  // velocity-cell edges for the bin searches: shared memory serves the
  // threads' different addresses in parallel (constant memory serialises)
  __shared__ double VE1[MAXV + 1], VE2[MAXV + 1], VEP[MAXV + 1];
  if (a.bin || !THREE_D) load_vgrid_smem(c_vg.e1, c_vg.e2, c_vg.epar, VE1, VE2, VEP);
  // one work item per block, or a persistent grid striding over the items
  for (int item = blockIdx.x; item < a.nitems; item += gridDim.x) {
  const int t = a.blk_tube[item];
  const int64_t nl = a.nlive[t];
  const int64_t beg = a.blk_start[item];
  if (beg >= nl) continue;  // idle chunk (uniform over the block)
  const int64_t end = min(beg + (int64_t)a.chunk, nl);
  __syncthreads();  // the previous item is done with the shared tables
  if (t != tcur) {
    load_tube_smem(a, t, T, E, Cc);
    tcur = t;
  }
  if (a.cxc)
    for (int k = threadIdx.x; k < T.nq; k += blockDim.x) HC[k] = 0u;
  BinWin W{};
  if (a.bin)
    W = bin_win_init(HC + nqmax, a.ion.qind[T.off + beg], T.nq);
  __syncthreads();
  const double ipG = 1.0 / T.pG, invsumds = 1.0 / T.sumdsICR;
  const double qs_ms = T.qs / T.ms;
  const double c_invOm = T.ms / (T.qs * MDIP);
  for (int64_t i = beg + threadIdx.x; i < end; i += blockDim.x) {
    const int64_t j = T.off + i;
    const int qprev = I.qind[j];
    if (qprev == DEAD) continue;
    const double rho = I.rho[j], z = I.z[j], vpar = I.vpar[j];
    double v1 = I.v1[j], v2 = I.v2[j];
    double aea = I.aea[j], ag = I.ag[j];
    if (a.prologue) field_prologue(a, T, E, Cc, I.qk4[j], qprev, aea, ag);
    // Vperp^2 without a fused multiply-add: its square root is the 2D grid's
    // binned speed (vperp_mag), the same value on every path
    const double vp2 = __dadd_rn(__dmul_rn(v1, v1), __dmul_rn(v2, v2));
    // ---- k1: KineticUpdateA -------------------------------------------
    const Geo<double> g1 = geo(rho, z);
    const int qi = cell_search_from(E, T.nq, T.sgn * g1.q, qprev);
    int b1 = -1, b2 = -1, bp = -1;
    if (THREE_D) {
      if (a.bin) {
        bp = vbin(VEP, c_vg.npar, vpar);
        b1 = vbin(VE1, c_vg.n1, v1);
        b2 = vbin(VE2, c_vg.n2, v2);
      }
    } else {  // 2D grid: an out-of-grid speed keeps its previous bin
      const int old = I.vb[j];
      const int np_ = vbin(VEP, c_vg.npar, vpar);
      const int n1_ = vbin(VE1, c_vg.n1, sqrt(vp2));
      bp = np_ >= 0 ? np_ : (old & 0xffff) - 1;
      b1 = n1_ >= 0 ? n1_ : (old >> 16) - 1;
      const int nw = ((b1 + 1) << 16) | (bp + 1);
      if (nw != old && !a.bin_only) I.vb[j] = nw;
    }
    if (a.bin) accumulate_win(a.acc, T, W, qi, b1, b2, bp, a.exporting);
    if (a.bin_only) {
      if (a.write_qind) I.qind[j] = qi;
      continue;
    }
    const double a1 = apar(g1, vp2, aea, ag, a.ff);
    // wave heating (the mirror force keeps the pre-kick Vperp)
    double v1n = v1, v2n = v2;
    if (a.icr && qi >= 0) {
      const double sl = g1.ell * g1.isl;
      const double Om = qs_ms * MDIP * sl * (g1.ir * g1.ir * g1.ir);
      const double r = 1.0 / g1.ir;
      const double invOm = c_invOm * (r * r * r) * g1.isl;
      const HeatC<double> hc = heat_consts<double>(a.ct, (int64_t)T.coff + qi);
      heat<double>(a, step, hc, I.id[j], invsumds, Om, invOm, fabs(vpar), v1n, v2n);
    }
    // ---- k2: half step along V_R (KineticUpdateB) -----------------------
    const double VRr = vpar * g1.er, VRz = vpar * g1.ez;
    const Geo<double> g2 = geo(fma(hh, VRr, rho), fma(hh, VRz, z));
    const double a2 = apar(g2, vp2, aea, ag, a.ff);
    // ---- k4: x + h V_R + h^2/2 A1 (KineticUpdateC) ----------------------
    const double A1r = a1 * g1.er, A1z = a1 * g1.ez;
    const Geo<double> g4 = geo(rho + h * VRr + hsq2 * A1r, z + h * VRz + hsq2 * A1z);
    const double a4 = apar(g4, vp2, aea, ag, a.ff);
    if (a.write_qk4) {
      I.qk4[j] = g4.q;
      if (I.rho4) {  // KineticUpdateC stores the k4 geometry for collisions
        I.rho4[j] = rho + h * VRr + hsq2 * A1r;
        I.z4[j] = z + h * VRz + hsq2 * A1z;
      }
    }
    const double A2r = a2 * g2.er, A2z = a2 * g2.ez;
    const double A4r = a4 * g4.er, A4z = a4 * g4.ez;
    // ---- RK combination (k3 = k2) ---------------------------------------
    const double VNr = VRr + h6 * (A1r + 2.0 * A2r + 2.0 * A2r + A4r);
    const double VNz = VRz + h6 * (A1z + 2.0 * A2z + 2.0 * A2z + A4z);
    const double Vk2r = VRr + hh * A1r, Vk2z = VRz + hh * A1z;
    const double Vk4r = VRr + h * A2r, Vk4z = VRz + h * A2z;
    const double xr = rho + h6 * (VRr + 2.0 * Vk2r + 2.0 * Vk2r + Vk4r);
    const double xz = z + h6 * (VRz + 2.0 * Vk2z + 2.0 * Vk2z + Vk4z);
    // ---- re-projection onto the tube: q of the RK point, p reset to pG --
    const double r2 = xr * xr + xz * xz;
    const double ir = rsqrt(r2);
    const double qN = (RE * RE) * (xz * ir) * (ir * ir);
    const double u = quartic_newton(qN, ipG, r2 * ir * (1.0 / RE), 2);
    const double s2 = u * ipG;                 // sin^2(theta)
    const double st = s2 * rsqrt(s2);
    const double ctn = qN * u * u;
    const double rr = u * RE;
    double rhoN = rr * st, zN = rr * ctn;
    if (fabs(rhoN) < 1e-6) rhoN = 0.0;
    if (fabs(zN) < 1e-6) zN = 0.0;
    // ---- V|| along the new field direction ------------------------------
    const double isl = rsqrt(1.0 + 3.0 * ctn * ctn);
    const double vparN = (3.0 * ctn * st * isl) * VNr + ((3.0 * ctn * ctn - 1.0) * isl) * VNz;
    if (!isfinite(vparN) || !isfinite(zN)) atomicOr(a.status, ST_NAN);
    I.rho[j] = rhoN;
    I.z[j] = zN;
    I.vpar[j] = vparN;
    if (a.icr) {
      I.v1[j] = v1n;
      I.v2[j] = v2n;
    }
    if (a.prologue) {
      I.aea[j] = aea;
      I.ag[j] = ag;
    }
    if (a.write_qind) I.qind[j] = qi;
    if (a.cxc && qi >= 0) atomicAdd(&HC[qi], 1u);
  }
  if (a.bin) bin_win_flush(a.acc, T, W);
  if (a.cxc) flush_cx_counts(a, t, beg, T.nq, HC);
  if (!PERSIST) break;  // one item per block: no loop-carried state
  }  // work items
}

// The force switches of apar as 0/1 factors for the mixed push: a|| =
// s (cm m - cg |AG| + ce2 |AEA|) + ce1 AEA without branches (the sign s = -1
// south of the equator).
struct ForceC {
  float cm, cg, ce1, ce2;  // mirror, gravity, signed / unsigned ambipolar
};
__device__ __forceinline__ ForceC force_c(const ForceFlags &f) {
  return ForceC{f.mirror ? 1.0f : 0.0f, f.grav ? 1.0f : 0.0f,
                (f.eamb && f.eambsign) ? 1.0f : 0.0f,
                (f.eamb && !f.eambsign) ? 1.0f : 0.0f};
}

// Start-of-step velocity bins of one ion from its FP64 velocities and the
// FP64 edges: (V⊥1, V⊥2, V∥) on the 3D grid; on the 2D grid (|V⊥|, V∥)
// with the previous bin kept for a value outside the grid (the stale-index
// rule), stored back when it changed.
template <bool THREE_D>
__device__ __forceinline__ void start_bins(const PushArgs &a, const Ions &I,
                                           int64_t j, const double *VE1,
                                           const double *VE2, const double *VEP,
                                           const VBinTab &VT1, const VBinTab &VT2,
                                           const VBinTab &VTP, double vpar,
                                           double v1, double v2, int &b1, int &b2,
                                           int &bp) {
  b2 = -1;
  if (THREE_D) {
    bp = vbin_tab(VTP, VEP, c_vg.npar, vpar);
    b1 = vbin_tab(VT1, VE1, c_vg.n1, v1);
    b2 = vbin_tab(VT2, VE2, c_vg.n2, v2);
  } else {
    const int old = I.vb[j];
    const int np_ = vbin_tab(VTP, VEP, c_vg.npar, vpar);
    const int n1_ = vbin_tab(VT1, VE1, c_vg.n1, vperp_mag(v1, v2));
    bp = np_ >= 0 ? np_ : (old & 0xffff) - 1;
    b1 = n1_ >= 0 ? n1_ : (old >> 16) - 1;
    const int nw = ((b1 + 1) << 16) | (bp + 1);
    if (nw != old && !a.bin_only) I.vb[j] = nw;
  }
}

// ---------------------------------------------------------------------------
// Mixed kernel: FP32 arithmetic on FP64 state.  The position is one FP64
// cell coordinate x = cell + offset in q within the cell; V|| and the Vperp
// pair are FP64.  Every RK stage, force evaluation and the heating kick run
// in FP32; FP64 is kept for the q reconstruction, the quartic root (Newton
// from a per-cell linear guess), the dominant displacement term h V|| e1,
// the renormalised q of the new position, the accumulation of the FP32
// velocity increments into the FP64 velocities, and all reductions.  The
// start-of-step bins compare the FP64 velocities with the FP64 edges, as
// the FP64 path does.
//
// V|| along the new field direction: with e1, e2, e4, eN the field
// directions at the start, k2, k4 and new points, the FP64 path computes
// eN . (V|| e1 + h/6 (a1 e1 + 4 a2 e2 + a4 e4)).  All of e1..e4 lie within
// ~1e-6 rad of eN, so e_k . eN = 1 - O(1e-12): the update is
//   V||N = V|| + h/6 (a1 + 4 a2 + a4) - V|| dal^2 / 2,
// dal = angle between e1 and eN = 3 (1 + cos^2) / (1 + 3 cos^2) dtheta along
// the dipole line (d/dtheta of atan2(3 cos sin, 3 cos^2 - 1)), an FP32
// increment added to the FP64 V||.
// NT threads per block and MINB resident blocks per SM set the register
// budget (256 x 4: 64 registers, 256 x 3: 80, 128 x 7: 72); the autotuner
// picks one.  K64 (precision mode KAOS_PREC_MIXED_K64) computes the heating
// kick in FP64 from the FP64 state, with the FP64 path's formula and Philox
// draw; the rest of the step is unchanged.
template <bool THREE_D, int NT, int MINB, bool PERSIST, bool MASTER, bool K64>
__global__ void __launch_bounds__(NT, MINB) k_push32(PushArgs a) {
  // master-step work (field re-interpolation, binning) only in the MASTER
  // variant: the ordinary step carries none of its code or registers
  const bool bin = MASTER && a.bin, prologue = MASTER && a.prologue,
             bin_only = MASTER && a.bin_only;
  extern __shared__ __align__(16) double sm[];
  const int nqmax = a.nqs;
  double *E = sm, *Cc = sm + nqmax + 1;
  double *UL = Cc + nqmax, *UD = UL + nqmax, *UC = UD + nqmax, *QL = UC + nqmax,
         *IDQ = QL + nqmax, *DQ = IDQ + nqmax;
  // 8 floats per cell (heat32), 16-byte aligned; then the cell fields
  // (EAmag, EG) of the field re-interpolation
  float *HK = (float *)(sm + ((8 * nqmax + 2) & ~1));
  float2 *FE = (float2 *)(HK + 8 * nqmax);
  unsigned *HC = (unsigned *)(FE + nqmax);
  const float h = (float)a.h, hh = 0.5f * h, h6 = h / 6.0f, hsq2 = 0.5f * h * h;
  const float hh6 = h * h6;
  const double hd = a.h;
  const uint32_t step = a.dstep ? *a.dstep : a.step;
  const float fRE = (float)RE;
  const ForceC fc = force_c(a.ff);
  Ions I = a.ion;
  TubeD T;
  int tcur = -1;
  // velocity-cell edges for the bin searches in shared memory (FP64 edges
  // for the comparisons, FP32 lookup tables for the first guess), after the
  // binning window; only the variants that bin are launched with room for
  // them (BINS_SMEM_BYTES)
  // (offset arithmetic from the shared array itself: a pointer rebuilt from
  // an integer would lose its address space and the searches would issue
  // generic loads)
  const size_t ve_off =
      ((size_t)((const char *)(HC + nqmax + bin_win_size()) - (const char *)sm) + 15) &
      ~(size_t)15;
  double *VE1 = (double *)((char *)sm + ve_off);
  double *VE2 = VE1 + (MAXV + 1), *VEP = VE2 + (MAXV + 1);
  VBinTab *VTS = (VBinTab *)(VEP + (MAXV + 1));
  VBinTab &VT1 = VTS[0], &VT2 = VTS[1], &VTP = VTS[2];
  if (K64) kf_tables_fill(kf_tables());  // ordered by the item loop's barrier
  if (bin || !THREE_D) {
    load_vgrid_smem(c_vg.e1, c_vg.e2, c_vg.epar, VE1, VE2, VEP);
    build_vbin_tab(VTP, c_vg.epar, c_vg.npar);
    build_vbin_tab(VT1, c_vg.e1, c_vg.n1);
    if (THREE_D) build_vbin_tab(VT2, c_vg.e2, c_vg.n2);
    // the first barrier of the item loop orders the tables before any use
  }
  // one work item per block, or a persistent grid striding over the items
  for (int item = blockIdx.x; item < a.nitems; item += gridDim.x) {
  const int t = a.blk_tube[item];
  const int64_t nl = a.nlive[t];
  const int64_t beg = a.blk_start[item];
  if (beg >= nl) continue;  // idle chunk (uniform over the block)
  const int64_t end = min(beg + (int64_t)a.chunk, nl);
  __syncthreads();  // the previous item is done with the shared tables
  if (t != tcur) {
    load_tube_smem(a, t, T, E, Cc);
    for (int k = threadIdx.x; k < T.nq; k += blockDim.x) {
      const int64_t g = T.coff + k;
      const double ql = a.ct.qGL[g], qh = a.ct.qGH[g];
      QL[k] = ql;
      DQ[k] = qh - ql;
      IDQ[k] = 1.0 / (qh - ql);
      UL[k] = a.ct.uL[g];
      UD[k] = a.ct.uH[g] - a.ct.uL[g];
      // quadratic in the offset through the edges and the midpoint
      UC[k] = 4.0 * a.ct.uM[g] - 2.0 * (a.ct.uL[g] + a.ct.uH[g]);
      if (a.icr) {
        const double lam = a.ct.lambdaPerp[g];
        HK[8 * k + 0] = (float)a.ct.hK1[g];
        HK[8 * k + 1] = (float)a.ct.hK2[g];
        HK[8 * k + 2] = (float)a.ct.hc1[g];
        HK[8 * k + 3] = (float)a.ct.hc2[g];
        HK[8 * k + 4] = a.icrcoh ? (float)a.ct.hiom0[g] : lg2f((float)a.ct.hiom0[g]);
        HK[8 * k + 5] = (float)lam;
        HK[8 * k + 6] = lam != 0.0 ? (float)log2(2.0 * PI / lam) : 0.0f;
        HK[8 * k + 7] = 0.0f;
      }
      if (prologue) FE[k] = make_float2((float)a.ct.EAmag[g], (float)a.ct.EG[g]);
    }
    tcur = t;
  }
  if (a.cxc)
    for (int k = threadIdx.x; k < T.nq; k += blockDim.x) HC[k] = 0u;
  BinWin W{};
  if (bin) {
    const double xf = a.ion.x[T.off + beg];
    W = bin_win_init(HC + nqmax, xf < XDEAD_LIM ? 0 : x_cell(xf, T.nq), T.nq);
  }
  __syncthreads();
  const float invsumds = (float)(1.0 / T.sumdsICR);
  const double ipG = 1.0 / T.pG;
  const float qs_ms = (float)(T.qs / T.ms);
  const float c_invOm = (float)(T.ms / (T.qs * MDIP));
  const float ylim = (float)((2.0 * PI / a.h) * (2.0 * PI / a.h));
  // the FP64 kick's per-tube constants (K64 only)
  const double qs_ms64 = T.qs / T.ms, c_invOm64 = T.ms / (T.qs * MDIP);
  const double invsumds64 = 1.0 / T.sumdsICR;
  const double ylim64 = (2.0 * PI / a.h) * (2.0 * PI / a.h);
  // the item's ions through per-item base pointers and a 32-bit index
  const int64_t base = T.off + beg;
  const int nk = (int)(end - beg);
  double *__restrict__ X = I.x + base;
  double *__restrict__ VP = I.vpar + base;
  double2 *__restrict__ V12 = I.v12 + base;
  float2 *__restrict__ FF = I.ffl + base;
  float *__restrict__ QK = I.fqk4 + base;
  int32_t *__restrict__ QI = I.qind + base;
  const uint64_t *__restrict__ ID = I.id + base;
  // Software pipeline: the state of the next ion of this thread is loaded
  // before the current one is pushed, so its HBM latency overlaps the work.
  double n_x = XDEAD, n_vp = 0.0;
  double2 n_v = make_double2(0.0, 0.0);
  float2 n_f = make_float2(0.f, 0.f);
  uint64_t n_id = 0;
  float n_qk = 0.f;  // q_k4 of the master-step field re-interpolation
  if ((int)threadIdx.x < nk) {
    const unsigned k = threadIdx.x;
    n_x = X[k];
    n_vp = VP[k];
    n_v = V12[k];
    n_f = FF[k];
    if (a.icr) n_id = ID[k];
    if (prologue) n_qk = QK[k];
  }
  for (unsigned k = threadIdx.x; k < (unsigned)nk; k += NT) {
    const int64_t j = base + k;  // the ion's slot (2D grid: its stale bins)
    const double x0 = n_x;
    const double vpar = n_vp;
    const double v1 = n_v.x, v2 = n_v.y;
    float aea = n_f.x, ag = n_f.y;
    const uint64_t pid = n_id;
    const float qk0 = n_qk;
    if (k + NT < (unsigned)nk) {
      const unsigned kn = k + NT;
      n_x = X[kn];
      n_vp = VP[kn];
      n_v = V12[kn];
      n_f = FF[kn];
      if (a.icr) n_id = ID[kn];
      if (prologue) n_qk = QK[kn];
    }
    if (x0 < XDEAD_LIM) continue;  // slot marked DEAD
    const int c0 = x_cell(x0, T.nq);
    const double o0 = x0 - (double)c0;  // exact
    if (prologue) field_prologue32(a.ff, T, E, Cc, FE, qk0, c0, qs_ms, aea, ag);
    // ---- start-of-step position: q, then (r, theta) by FP64 Newton -------
    const double q0 = fma(o0, DQ[c0], QL[c0]);
    // per-cell quadratic guess u(o) = uL + o (uH - uL) + o (1 - o) UC
    const double u = quartic_newton_chord(
        q0, ipG, fma(o0, fma(1.0 - o0, UC[c0], UD[c0]), UL[c0]));
    const double s2 = u * ipG;  // sin^2(theta)
    // sqrt(s2): FP32 seed and one FP64 Newton step (relative error ~1e-14)
    const float s2f = (float)s2;
    const float ysf = rsq(s2f);
    double ys = (double)ysf;
    ys = ys * fma(-0.5 * s2 * ys, ys, 1.5);
    const double st = s2 * ys;
    const double ct = q0 * u * u;
    const double r = u * RE;
    const double rho0 = r * st, z0 = r * ct;
    // an offset strictly inside (0, 1) puts q0 inside cell c0 (its FP64
    // rounding is far below the margin): no edge search
    const int qi = (o0 > 1e-9 && o0 < 1.0 - 1e-9)
                       ? c0 : cell_search_from(E, T.nq, T.sgn * q0, c0);
    // ---- k1 geometry in FP32, from FP32 values (cos = q u^2, sin = s2
    // rsqrt(s2)): two FP64->FP32 conversions fewer on the busy XU pipe, for
    // a few FP32 roundings in forces that carry FP32 rounding anyway -------
    Geo<float> g1;
    g1.q = (float)q0;
    const float uf = (float)u;
    g1.ct = g1.q * uf * uf;
    g1.st = s2f * ysf;
    const float rfl = uf * fRE;  // r in FP32
    g1.ir = rcpa(rfl);
    g1.ell = 1.0f + 3.0f * g1.ct * g1.ct;
    g1.isl = rsq(g1.ell);
    g1.er = 3.0f * g1.ct * g1.st * g1.isl;
    g1.ez = (3.0f * g1.ct * g1.ct - 1.0f) * g1.isl;
    const float vparf = (float)vpar, v1f = (float)v1, v2f = (float)v2;
    const float vp2 = v1f * v1f + v2f * v2f;
    // the FP32 meridian point (used for the k2/k4 hemisphere signs and the
    // turn of the field direction) from values already in FP32
    const float rf = g1.st * rfl, zf = g1.ct * rfl;
    // ---- the dominant displacement term h V|| e1 in FP64 (the direction
    // from the FP64 cos/sin, 1/sqrt(ell) from the FP32 value and one FP64
    // Newton step), taken now so that only its end point stays live --------
    const double ell64 = fma(3.0 * ct, ct, 1.0);
    double yl = (double)g1.isl;
    yl = yl * fma(-0.5 * ell64 * yl, yl, 1.5);
    const double hv = hd * vpar * yl;
    const double xr0 = fma(hv, 3.0 * ct * st, rho0);
    const double xz0 = fma(hv, fma(3.0 * ct, ct, -1.0), z0);
    if (bin_only) {
      int b1, b2, bp;
      start_bins<THREE_D>(a, I, j, VE1, VE2, VEP, VT1, VT2, VTP, vpar, v1, v2, b1, b2, bp);
      if (bin) accumulate_win(a.acc, T, W, qi, b1, b2, bp, a.exporting);
      if (a.write_qind) QI[k] = qi;
      continue;
    }
    double v1n = v1, v2n = v2;  // after the wave-heating kick
    // (the FP64 kick of K64 runs after the position and V|| stores below:
    // nothing before them reads the kicked pair)
    if (!K64 && a.icr && qi >= 0) {
      const float rr = (float)r;
      const float sl = g1.ell * g1.isl;
      const float ir3 = g1.ir * g1.ir * g1.ir;
      const float Om = qs_ms * (float)MDIP * sl * ir3;
      const float *hk = HK + 8 * qi;
      if (!a.icrcoh) {
        float dv1, dv2;
        heat32(a, step, hk, pid, invsumds, ylim, Om, fabsf(vparf), vp2, dv1, dv2);
        v1n = v1 + (double)dv1;
        v2n = v2 + (double)dv2;
      } else {
        const float invOm = c_invOm * (rr * rr * rr) * g1.isl;
        const HeatC<float> hc{hk[0], hk[1], hk[2], hk[3], hk[4], hk[5]};
        float w1 = v1f, w2 = v2f;
        heat<float>(a, step, hc, pid, invsumds, Om, invOm, fabsf(vparf), w1, w2);
        v1n = (double)w1;
        v2n = (double)w2;
      }
    }
    // stored at once: the kicked pair holds no registers through the RK
    if (!K64 && a.icr) V12[k] = make_double2(v1n, v2n);
    // ---- the stage accelerations ----------------------------------------
    // a|| = M + s C0 + ce1 AEA with the signed mirror term M (cos(theta) in
    // place of s |cos|: smooth through the equator), the hemisphere sign s
    // and the per-ion constant C0 = -|AG| + |AEA| (gravity and the unsigned
    // ambipolar field; the cached fields do not change within a step).  The
    // k2 and k4 points lie on the line x1 + ds e1 (|ds| = |V|| h| + ... is
    // below ~300 m against a length scale r/3 > 2e6 m), so M there is
    // M1 + dM/ds ds to a relative 1e-8 (1e-12 at the typical 10 m), below
    // the FP32 rounding; with F = cos (2 + sin^2/ell) / (r sqrt(ell)),
    // dF/ds = [s^2 c^2 (8 + 9 s^2/ell)/ell - (1 + c^2)(2 + s^2/ell)] / (ell r^2)
    // (dr/ds = 2c/sqrt(ell), dtheta/ds = s/(r sqrt(ell)) along the dipole e).
    const float il = g1.isl * g1.isl;  // 1/ell
    const float sn2 = g1.st * g1.st, cs2 = g1.ct * g1.ct;
    const float G2 = fmaf(sn2, il, 2.0f);
    const float hm = fc.cm * 1.5f * vp2 * g1.ir;
    const float M1 = hm * g1.ct * G2 * g1.isl;
    const float dM = hm * g1.ir * il *
                     fmaf(sn2 * cs2 * il, fmaf(9.0f * sn2, il, 8.0f), -(1.0f + cs2) * G2);
    const float C0 = fc.ce2 * fabsf(aea) - fc.cg * fabsf(ag);
    const float Ce = fc.ce1 * aea;
    const float a1 = M1 + (g1.ct <= 0.0f ? -C0 : C0) + Ce;
    const float VRr = vparf * g1.er, VRz = vparf * g1.ez;
    const float ds2 = hh * vparf, ds4 = fmaf(hsq2, a1, h * vparf);
    const float z2 = fmaf(ds2, g1.ez, zf), z4 = fmaf(ds4, g1.ez, zf);
    const float a2 = fmaf(dM, ds2, M1) + (z2 <= 0.0f ? -C0 : C0) + Ce;
    const float a4 = fmaf(dM, ds4, M1) + (z4 <= 0.0f ? -C0 : C0) + Ce;
    // q at the k4 point: dq/ds = -RE^2 sqrt(ell) / r^3 along e1
    if (a.write_qk4)
      QK[k] = fmaf(-(float)(RE * RE) * (g1.ell * g1.isl) * (g1.ir * g1.ir * g1.ir), ds4, g1.q);
    // ---- displacement h/6 (V_R + 4 (V_R + h/2 A1) + (V_R + h A2)) ---------
    // = h V|| e1 (FP64, above) + h^2/6 (2 a1 + a2) e1 (FP32; the k2 point's
    // direction differs from e1 by ~1e-6 rad, ~1e-10 m here)
    const float ac = hh6 * (2.0f * a1 + a2);
    const float ddr = ac * g1.er, ddz = ac * g1.ez;
    // ---- renormalisation in FP64: q of the new point --------------------
    const double xr = xr0 + (double)ddr, xz = xz0 + (double)ddz;
    const double r2 = xr * xr + xz * xz;
    double y = (double)rsq((float)r2);
    y = y * fma(-0.5 * r2 * y, y, 1.5);
    const double qN = (RE * RE) * xz * (y * y * y);
    // the new cell: most ions stay in the cell they started the step in,
    // and an offset strictly inside (0, 1) there decides it without the
    // edge search; escaped ions keep the end cell and an offset outside
    const int cs = qi >= 0 ? qi : c0;
    double od = (qN - QL[cs]) * IDQ[cs];
    int cpos = cs;
    if (!(od > 1e-9 && od < 1.0 - 1e-9)) {
      const int cN = cell_search_from(E, T.nq, T.sgn * qN, cs);
      cpos = cN >= 0 ? cN : (cN == BELOW ? 0 : T.nq - 1);
      od = (qN - QL[cpos]) * IDQ[cpos];
    }
    const double xN = (double)cpos + od;
    // ---- V|| along the new field direction ------------------------------
    const float dth = (zf * fmaf(h, VRr, ddr) - rf * fmaf(h, VRz, ddz)) * (g1.ir * g1.ir);
    const float dal = 3.0f * fmaf(g1.ct, g1.ct, 1.0f) * (g1.isl * g1.isl) * dth;
    const float dv = fmaf(h6, a1 + 4.0f * a2 + a4, -0.5f * vparf * dal * dal);
    const double vparN = vpar + (double)dv;
    if (bin || !THREE_D) {
      int b1, b2, bp;
      start_bins<THREE_D>(a, I, j, VE1, VE2, VEP, VT1, VT2, VTP, vpar, v1, v2, b1, b2, bp);
      if (bin) accumulate_win(a.acc, T, W, qi, b1, b2, bp, a.exporting);
    }
    if (!isfinite(vparN) || !isfinite(xN)) atomicOr(a.status, ST_NAN);
    X[k] = xN;
    VP[k] = vparN;
    if (prologue) FF[k] = make_float2(aea, ag);
    if (a.write_qind) QI[k] = qi;
    if (a.cxc && qi >= 0) atomicAdd(&HC[qi], 1u);
    if (K64 && a.icr) {
      if (qi >= 0) {
        // FP64 kick at the start-of-step point: Omega = (q/m) MDIP sqrt(ell)
        // / r^3 and 1/Omega from the FP64 radius and 1/sqrt(ell) (yl), 1/r
        // from the FP32 reciprocal and one FP64 Newton step (relative error
        // ~1e-14); the RK above used the pre-kick Vperp, as heat() does
        double ir = (double)rcpa((float)r);
        ir = ir * fma(-r, ir, 2.0);
        const double Om = qs_ms64 * MDIP * (ell64 * yl) * (ir * ir * ir);
        const double invOm = c_invOm64 * (r * r * r) * yl;
        if (!a.icrcoh) {
          heat64t(a, step, kf_tables(), a.ct, (int64_t)T.coff + qi, pid, invsumds64,
                  ylim64, Om, invOm, fabs(vpar), v1n, v2n);
        } else {  // coherent branch: the FP64 path's own code
          const HeatC<double> hc = heat_consts<double>(a.ct, (int64_t)T.coff + qi);
          heat<double>(a, step, hc, pid, invsumds64, Om, invOm, fabs(vpar), v1n, v2n);
        }
      }
      V12[k] = make_double2(v1n, v2n);
    }
  }
  if (bin) bin_win_flush(a.acc, T, W);
  if (a.cxc) flush_cx_counts(a, t, beg, T.nq, HC);
  if (!PERSIST) break;  // one item per block: no loop-carried state
  }  // work items
}

}  // namespace kaos
