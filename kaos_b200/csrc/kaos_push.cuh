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

namespace kaos {

__constant__ VGridC c_vg;

struct PushArgs {
  const TubeD *tubes;
  const int *blk_tube;
  const int64_t *blk_start;
  int chunk;
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
};

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
  if (exporting) {
    int64_t nv = d3 ? (int64_t)c_vg.n1 * c_vg.n2 * c_vg.npar
                    : (int64_t)c_vg.n1 * c_vg.npar;
    int64_t b = d3 ? ((int64_t)b1 * c_vg.n2 + b2) * c_vg.npar + bp
                   : (int64_t)b1 * c_vg.npar + bp;
    atomicAdd(acc.hist + T.hoff + (int64_t)qi * nv + b, 1u);
  }
}

// Field magnitude at q by linear interpolation between cell centres with
// constant half cells at both ends (_8_7_AmbipolarEfield.f90:1453-2722);
// returns false outside the grid (the particle keeps its value).
__device__ __forceinline__ bool interp_centres(const double *E, const double *C,
                                               const double *Eg,
                                               const double *qC, int nq,
                                               double sgn, double q,
                                               double *out) {
  double s = sgn * q;
  if (s < E[0] || s > E[nq]) return false;
  if (s <= C[0]) { *out = Eg[0]; return true; }
  if (s >= C[nq - 1]) { *out = Eg[nq - 1]; return true; }
  int lo = 1, hi = nq - 1;  // smallest k with s <= C[k]
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (s <= C[mid]) hi = mid; else lo = mid + 1;
  }
  double x1 = qC[lo - 1], x2 = qC[lo];
  *out = Eg[lo - 1] + (((q - x1) / (x2 - x1)) * (Eg[lo] - Eg[lo - 1]));
  return true;
}

__device__ __forceinline__ void field_prologue(const PushArgs &a,
                                               const TubeD &T, const double *E,
                                               const double *C, double qk,
                                               double &aea, double &ag) {
  const double qm = a.qs / a.ms;
  double v;
  if (a.ff.eamb && interp_centres(E, C, a.ct.EAmag + T.coff, a.ct.qGC + T.coff,
                                  T.nq, T.sgn, qk, &v)) {
    double e = a.ff.eambsign ? v : fabs(v);
    aea = (e == 0.0) ? 0.0 : (a.ff.eambsign ? qm * e : fabs(qm * e));
  }
  if (a.ff.grav && interp_centres(E, C, a.ct.EG + T.coff, a.ct.qGC + T.coff,
                                  T.nq, T.sgn, qk, &v)) {
    double e = fabs(v);
    ag = (e == 0.0) ? 0.0 : fabs(qm * e);
  }
}

// Box-Muller Gaussian from one Philox draw (GaussianRNGSub
// _3_1_GaussianRNG.f90:33); the FP32 variant transforms the same uniforms.
__device__ __forceinline__ double gauss64(uint64_t seed, uint64_t id,
                                          uint32_t step, uint32_t stream,
                                          uint32_t sub) {
  kaos_u32x4 w = kaos_philox((uint32_t)id, (uint32_t)(id >> 32), step,
                             (stream << 24) | sub, seed);
  double u1 = kaos_u01(w.v[0], w.v[1]);
  double u2 = kaos_u01(w.v[2], w.v[3]);
  return sqrt(-2.0 * log(u1)) * cos(2.0 * PI * u2);
}
__device__ __forceinline__ float gauss32(uint64_t seed, uint64_t id,
                                         uint32_t step, uint32_t stream,
                                         uint32_t sub) {
  kaos_u32x4 w = kaos_philox((uint32_t)id, (uint32_t)(id >> 32), step,
                             (stream << 24) | sub, seed);
  float u1 = (float)kaos_u01(w.v[0], w.v[1]);
  float u2 = (float)kaos_u01(w.v[2], w.v[3]);
  return sqrtf(-2.0f * __logf(u1)) * __cosf(6.2831853071795865f * u2);
}

// WaveHeatingSub stochastic / coherent kicks (_8_1_1_0_WaveHeating.f90:
// 39-312) for an ion in valid cell gc with gyrofrequency Om at k1.
template <typename T>
__device__ __forceinline__ void heat(const PushArgs &a, int64_t gc, uint64_t id,
                                     double sumds, T Om, T vparabs, T &v1,
                                     T &v2) {
  const CellTables &c = a.ct;
  const bool f64 = sizeof(T) == 8;
  T lam = (T)c.lambdaPerp[gc], eta = (T)c.EtaLH[gc], xi1 = (T)c.XiPerp1[gc],
    xi2 = (T)c.XiPerp2[gc], Om0 = (T)c.OmegaG0[gc],
    chi1 = (T)c.ChiPerp1[gc], chi2 = (T)c.ChiPerp2[gc];
  const T h = (T)a.h, twopi = (T)(2.0 * PI);
  T vpm = sqrt(v1 * v1 + v2 * v2);
  T Sig = T(1);
  if (lam != T(0) && ((twopi * vpm) / Om) >= lam) Sig = (twopi * vpm) / (lam * Om);
  // q^2/(2 m^2) S0 in FP64: m^2 (~1e-51 kg^2) is below the FP32 range
  T pre = (T)((a.qs * a.qs / (2.0 * a.ms * a.ms)) * c.S0[gc]);
  T sig3 = (Sig == T(1)) ? T(1) : T(1) / (Sig * Sig * Sig);
  T p1, p2;
  if (f64) {
    p1 = (T)pow((double)(Om / Om0), -(double)chi1);
    p2 = (T)pow((double)(Om / Om0), -(double)chi2);
  } else {
    float lr = __log2f((float)(Om / Om0));
    p1 = (T)exp2f(-(float)chi1 * lr);
    p2 = (T)exp2f(-(float)chi2 * lr);
  }
  T D1 = (pre * (xi1 * eta) * p1) * sig3;
  T D2 = (pre * (xi2 * eta) * p2) * sig3;
  // epsilon = |V_R| / (Omega * sum ds_ICR); tau = 1/((Omega/2pi) sqrt(eps))
  T eps = vparabs / (Om * (T)sumds);
  T tau = T(1) / ((Om / twopi) * sqrt(eps));
  T G1 = f64 ? (T)gauss64(a.seed, id, a.step, KAOS_RNG_HEAT, 0)
             : (T)gauss32(a.seed, id, a.step, KAOS_RNG_HEAT, 0);
  if (a.icrcoh) {
    T dV = h * sqrt(T(2) * (D1 + D2) / tau) * G1;
    T vpn = fabs(vpm + dV);
    kaos_u32x4 w = kaos_philox((uint32_t)id, (uint32_t)(id >> 32), a.step,
                               (KAOS_RNG_HEAT << 24) | 2u, a.seed);
    T ga = (T)kaos_u01(w.v[0], w.v[1]) * twopi;
    v1 = vpn * cos(ga);
    v2 = vpn * sin(ga);
    return;
  }
  T G2 = f64 ? (T)gauss64(a.seed, id, a.step, KAOS_RNG_HEAT, 1)
             : (T)gauss32(a.seed, id, a.step, KAOS_RNG_HEAT, 1);
  if (h <= tau) {  // (h/tau) sqrt(2 D tau) written as h sqrt(2 D / tau)
    v1 = v1 + h * sqrt(T(2) * D1 / tau) * G1;
    v2 = v2 + h * sqrt(T(2) * D2 / tau) * G2;
  }
}

// Positive root u = r/RE of q^2 u^4 + u/p - 1 = 0 by Newton from u0 (the
// function is increasing and convex for u > 0, so the root is unique).
__device__ __forceinline__ double quartic_newton(double q, double p, double u,
                                                 int iters) {
  double q2 = q * q, ip = 1.0 / p;
  for (int k = 0; k < iters; ++k) {
    double u2 = u * u;
    double f = fma(q2 * u2, u2, fma(u, ip, -1.0));
    double fp = fma(4.0 * q2 * u2, u, ip);
    u = u - f / fp;
  }
  return u;
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
  __syncthreads();
}

// ---------------------------------------------------------------------------
// FP64 kernel: ions stored as meridian-plane (rho, z) in FP64.
template <bool THREE_D>
__global__ void __launch_bounds__(256) k_push64(PushArgs a) {
  extern __shared__ double sm[];
  const int t = a.blk_tube[blockIdx.x];
  TubeD T;
  const int nqmax = a.tubes[t].nq;
  double *E = sm, *Cc = sm + nqmax + 1;
  load_tube_smem(a, t, T, E, Cc);
  const int64_t nl = a.nlive[t];
  const int64_t beg = a.blk_start[blockIdx.x];
  const int64_t end = min(beg + (int64_t)a.chunk, nl);
  const double h = a.h, hh = 0.5 * a.h, h6 = a.h / 6.0;
  const double qs_ms = a.qs / a.ms;
  Ions I = a.ion;
  for (int64_t i = beg + threadIdx.x; i < end; i += blockDim.x) {
    const int64_t j = T.off + i;
    const int qprev = I.qind[j];
    if (qprev == DEAD) continue;
    double rho = I.rho[j], z = I.z[j], vpar = I.vpar[j];
    double v1 = I.v1[j], v2 = I.v2[j];
    double aea = I.aea[j], ag = I.ag[j];
    if (a.prologue) field_prologue(a, T, E, Cc, I.qk4[j], aea, ag);
    const double vp2 = v1 * v1 + v2 * v2;
    // ---- k1: KineticUpdateA -------------------------------------------
    Geo<double> g1 = geo(rho, z);
    const int qi = cell_search(E, T.nq, T.sgn * g1.q);
    // velocity bins at k1 (stale-index rule of the 2D grid kept in vb)
    int b1 = -1, b2 = -1, bp = -1;
    if (THREE_D) {
      if (a.bin) {
        bp = vbin(c_vg.epar, c_vg.npar, vpar);
        b1 = vbin(c_vg.e1, c_vg.n1, v1);
        b2 = vbin(c_vg.e2, c_vg.n2, v2);
      }
    } else {
      const int old = I.vb[j];
      int np_ = vbin(c_vg.epar, c_vg.npar, vpar);
      int n1_ = vbin(c_vg.e1, c_vg.n1, sqrt(vp2));
      bp = np_ >= 0 ? np_ : (old & 0xffff) - 1;
      b1 = n1_ >= 0 ? n1_ : (old >> 16) - 1;
      const int nw = ((b1 + 1) << 16) | (bp + 1);
      if (nw != old && !a.bin_only) I.vb[j] = nw;
    }
    if (a.bin) accumulate(a.acc, T, qi, b1, b2, bp, a.exporting);
    if (a.bin_only) {
      if (a.write_qind) I.qind[j] = qi;
      continue;
    }
    const double a1 = apar(g1, vp2, aea, ag, a.ff);
    // wave heating (uses Vperp before the kick for the mirror force)
    double v1n = v1, v2n = v2;
    if (a.icr && qi >= 0) {
      const double B = MDIP * (g1.ell * g1.isl) * (g1.ir * g1.ir * g1.ir);
      heat<double>(a, (int64_t)T.coff + qi, I.id[j], T.sumdsICR, qs_ms * B,
                   fabs(vpar), v1n, v2n);
    }
    // ---- k2: half step along V_R (KineticUpdateB) -----------------------
    const double VRr = vpar * g1.er, VRz = vpar * g1.ez;
    Geo<double> g2 = geo(rho + hh * VRr, z + hh * VRz);
    const double a2 = apar(g2, vp2, aea, ag, a.ff);
    // ---- k4: x + h V_R + h^2/2 A1 (KineticUpdateC) ----------------------
    const double A1r = a1 * g1.er, A1z = a1 * g1.ez;
    Geo<double> g4 = geo(rho + h * VRr + (0.5 * h * h) * A1r,
                         z + h * VRz + (0.5 * h * h) * A1z);
    const double a4 = apar(g4, vp2, aea, ag, a.ff);
    if (a.write_qk4) I.qk4[j] = g4.q;
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
    const double u = quartic_newton(qN, T.pG, r2 * ir * (1.0 / RE), 3);
    const double st = sqrt(u / T.pG);
    const double ctn = qN * u * u;
    const double r = u * RE;
    double rhoN = r * st, zN = r * ctn;
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
  }
}

// ---------------------------------------------------------------------------
// Mixed kernel: position = (cell, FP32 offset in q); FP32 velocities and RK
// stages; FP64 for the q reconstruction, the quartic root (Newton, table
// guess) and the renormalised q of the new position.
template <bool THREE_D>
__global__ void __launch_bounds__(256) k_push32(PushArgs a) {
  extern __shared__ double sm[];
  const int t = a.blk_tube[blockIdx.x];
  TubeD T;
  const int nqmax = a.tubes[t].nq;
  double *E = sm, *Cc = sm + nqmax + 1;
  double *UL = Cc + nqmax, *UD = UL + nqmax, *QL = UD + nqmax, *DQ = QL + nqmax;
  load_tube_smem(a, t, T, E, Cc);
  for (int k = threadIdx.x; k < T.nq; k += blockDim.x) {
    const double ql = a.ct.qGL[T.coff + k], qh = a.ct.qGH[T.coff + k];
    QL[k] = ql;
    DQ[k] = qh - ql;
    UL[k] = a.ct.uL[T.coff + k];
    UD[k] = a.ct.uH[T.coff + k] - a.ct.uL[T.coff + k];
  }
  __syncthreads();
  const int64_t nl = a.nlive[t];
  const int64_t beg = a.blk_start[blockIdx.x];
  const int64_t end = min(beg + (int64_t)a.chunk, nl);
  const float h = (float)a.h, hh = 0.5f * h, h6 = h / 6.0f;
  const float hsq2 = 0.5f * h * h;
  const double qs_ms = a.qs / a.ms;
  const double pG = T.pG, ipG = 1.0 / T.pG;
  Ions I = a.ion;
  for (int64_t i = beg + threadIdx.x; i < end; i += blockDim.x) {
    const int64_t j = T.off + i;
    const int qprev = I.qind[j];
    if (qprev == DEAD) continue;
    const int c0 = I.cell[j];
    const float o0 = I.off[j];
    float vpar = I.fvpar[j], v1 = I.fv1[j], v2 = I.fv2[j];
    float aea = I.faea[j], ag = I.fag[j];
    if (a.prologue) {
      double da = aea, dg = ag;
      field_prologue(a, T, E, Cc, (double)I.fqk4[j], da, dg);
      aea = (float)da;
      ag = (float)dg;
    }
    // ---- start-of-step position: q, then (r, theta) by FP64 Newton -------
    const double q0 = QL[c0] + (double)o0 * DQ[c0];
    const double ug = UL[c0] + (double)o0 * UD[c0];
    const double u = quartic_newton(q0, pG, ug, 2);
    const double s2 = u * ipG;                       // sin^2(theta)
    float sf = sqrtf((float)s2);
    const double st = (double)sf + (s2 - (double)sf * sf) * (0.5 / (double)sf);
    const double ct = q0 * u * u;
    const double r = u * RE;
    const double rho0 = r * st, z0 = r * ct;
    const int qi = cell_search(E, T.nq, T.sgn * q0);
    // ---- k1 geometry in FP32 ---------------------------------------------
    Geo<float> g1;
    g1.ct = (float)ct;
    g1.st = (float)st;
    g1.ir = (float)(1.0 / r);
    g1.q = (float)q0;
    g1.ell = 1.0f + 3.0f * g1.ct * g1.ct;
    g1.isl = rsqrtf(g1.ell);
    g1.er = 3.0f * g1.ct * g1.st * g1.isl;
    g1.ez = (3.0f * g1.ct * g1.ct - 1.0f) * g1.isl;
    const float vp2 = v1 * v1 + v2 * v2;
    int b1 = -1, b2 = -1, bp = -1;
    if (THREE_D) {
      if (a.bin) {
        bp = vbin(c_vg.fpar, c_vg.npar, vpar);
        b1 = vbin(c_vg.f1, c_vg.n1, v1);
        b2 = vbin(c_vg.f2, c_vg.n2, v2);
      }
    } else {
      const int old = I.vb[j];
      int np_ = vbin(c_vg.fpar, c_vg.npar, vpar);
      int n1_ = vbin(c_vg.f1, c_vg.n1, sqrtf(vp2));
      bp = np_ >= 0 ? np_ : (old & 0xffff) - 1;
      b1 = n1_ >= 0 ? n1_ : (old >> 16) - 1;
      const int nw = ((b1 + 1) << 16) | (bp + 1);
      if (nw != old && !a.bin_only) I.vb[j] = nw;
    }
    if (a.bin) accumulate(a.acc, T, qi, b1, b2, bp, a.exporting);
    if (a.bin_only) {
      if (a.write_qind) I.qind[j] = qi;
      continue;
    }
    const float a1 = apar(g1, vp2, aea, ag, a.ff);
    float v1n = v1, v2n = v2;
    if (a.icr && qi >= 0) {
      const float B = (float)MDIP * (g1.ell * g1.isl) * (g1.ir * g1.ir * g1.ir);
      heat<float>(a, (int64_t)T.coff + qi, I.id[j], T.sumdsICR,
                  (float)qs_ms * B, fabsf(vpar), v1n, v2n);
    }
    const float rf = (float)rho0, zf = (float)z0;
    const float VRr = vpar * g1.er, VRz = vpar * g1.ez;
    Geo<float> g2 = geo(rf + hh * VRr, zf + hh * VRz);
    const float a2 = apar(g2, vp2, aea, ag, a.ff);
    const float A1r = a1 * g1.er, A1z = a1 * g1.ez;
    Geo<float> g4 = geo(rf + h * VRr + hsq2 * A1r, zf + h * VRz + hsq2 * A1z);
    const float a4 = apar(g4, vp2, aea, ag, a.ff);
    if (a.write_qk4) I.fqk4[j] = g4.q;
    const float A2r = a2 * g2.er, A2z = a2 * g2.ez;
    const float A4r = a4 * g4.er, A4z = a4 * g4.ez;
    const float VNr = VRr + h6 * (A1r + 4.0f * A2r + A4r);
    const float VNz = VRz + h6 * (A1z + 4.0f * A2z + A4z);
    // displacement h/6 (V_R + 4 (V_R + h/2 A1) + (V_R + h A2)) in FP32
    const float dr = h6 * (6.0f * VRr + 2.0f * h * A1r + h * A2r);
    const float dz = h6 * (6.0f * VRz + 2.0f * h * A1z + h * A2z);
    // ---- renormalisation in FP64: q of the new point --------------------
    const double xr = rho0 + (double)dr, xz = z0 + (double)dz;
    const double r2 = xr * xr + xz * xz;
    double y = (double)rsqrtf((float)r2);
    y = y * (1.5 - 0.5 * r2 * y * y);
    const double qN = (RE * RE) * xz * (y * y * y);
    int cN = cell_search(E, T.nq, T.sgn * qN);
    const int cpos = cN >= 0 ? cN : (cN == BELOW ? 0 : T.nq - 1);
    const float oN = (float)((qN - QL[cpos]) / DQ[cpos]);
    // ---- V|| along the new field direction (FP32) -----------------------
    Geo<float> gN = geo((float)xr, (float)xz);
    const float vparN = gN.er * VNr + gN.ez * VNz;
    if (!isfinite(vparN) || !isfinite(oN)) atomicOr(a.status, ST_NAN);
    I.cell[j] = cpos;
    I.off[j] = oN;
    I.fvpar[j] = vparN;
    if (a.icr) {
      I.fv1[j] = v1n;
      I.fv2[j] = v2n;
    }
    if (a.prologue) {
      I.faea[j] = aea;
      I.fag[j] = ag;
    }
    if (a.write_qind) I.qind[j] = qi;
  }
}

}  // namespace kaos
