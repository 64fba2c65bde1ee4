// kaos_tube.cuh -- per-tube and bookkeeping kernels of a master step:
// moments from the binning marginals, moment filter + ambipolar field +
// gravity field, ion-neutral collision counts, order-preserving removal of
// escaped ions and lower/upper-boundary injection.
#pragma once
#include "kaos_push.cuh"

namespace kaos {

struct TubeArgs {
  const TubeD *tubes;
  int ntubes;
  CellTables ct;
  Accum acc;
  const int64_t *nlive;
  double ms, qs, h, mNeut, TNeut, dNTe, dNTeEND;
  uint64_t seed;
  uint32_t nn;          // master-step index (reference nn)
  const uint32_t *dstep;  // graph replay: nn = step / ndatfac + 1 from device
  int ndatfac;
  int three_d;
  int te_update, have_import, eamb, grav, eapressure, eambsign, eambself,
      momfilter, qexchange, cenpar, cenperp;
  int fpM0, fpM1par, fpM1p1, fpM1p2, fpM2par;
};

// MomentFilterSub (_8_7_1_MomentFilter.f90:30-142) for cell Q of nq, input
// in shared memory.
__device__ double filter_cell(const double *in, int nq, int Q, int Pt) {
  const int H = (Pt - 1) / 2;
  const int LB = 0, UB = nq - 1;
  double out = 0.0;
  if (Q <= LB - 1 + H) {
    double s1 = in[Q] + in[Q + 1];
    for (int k = 2; k <= H; ++k) s1 += in[Q + k];
    double a1 = s1 / (H + 1);
    if (Q == LB) out = a1;
    else if (Q == LB + 1) out = (a1 + in[LB]) / 2.0;
    else {
      double s2 = in[Q - 1];
      for (int k = 2; k <= Q - LB; ++k) s2 += in[Q - k];
      out = (a1 + s2 / (Q - LB)) / 2.0;
    }
  }
  if ((Q > LB - 1 + H) && (Q < UB - H)) {
    double s1 = in[Q] + in[Q + 1];
    for (int k = 2; k <= H; ++k) s1 += in[Q + k];
    double s2 = in[Q - 1];
    for (int k = 2; k <= H; ++k) s2 += in[Q - k];
    out = (s1 / (H + 1) + s2 / H) / 2.0;
  }
  if (Q >= UB - H) {
    double s2 = in[Q] + in[Q - 1];
    for (int k = 2; k <= H; ++k) s2 += in[Q - k];
    double a2 = s2 / (H + 1);
    if (Q == UB) out = a2;
    else if (Q == UB - 1) out = (in[UB] + a2) / 2.0;
    else {
      double s1 = in[Q + 1];
      for (int k = 2; k <= UB - Q; ++k) s1 += in[Q + k];
      out = (s1 / (UB - Q) + a2) / 2.0;
    }
  }
  return out;
}

// ---------------------------------------------------------------------------
// AmbipolarEfieldSub pressure term (_8_7_AmbipolarEfield.f90:611-1299),
// GravfieldSub (_8_7_2_Gravfield.f90:57-65) and the Te update of
// KineticSolverSub (_8_KineticSolver.f90:69-89).  One block per tube.
__global__ void k_fields(TubeArgs a) {
  extern __shared__ double sm[];
  const TubeD T = a.tubes[blockIdx.x];
  const int nq = T.nq;
  double *M0p = sm, *M0f = sm + nq, *EP = sm + 2 * nq;
  const CellTables &c = a.ct;
  for (int Q = threadIdx.x; Q < nq; Q += blockDim.x) {
    const int64_t g = T.coff + Q;
    if (a.te_update) {
      double tn = c.Te[g] + a.dNTe;
      if (tn <= a.dNTeEND) c.Te[g] = tn;
    }
    M0p[Q] = c.M0prev[g];
    c.EG[g] = a.grav ? (-2.0 * GG * ME * T.ms * cos(c.thetaGC[g]) /
                        (T.qs * (c.rGC[g] * c.rGC[g]) * sqrt(c.ellGC[g])))
                     : 0.0;
  }
  __syncthreads();
  // the field rows of the moment block hold the fields last computed (read
  // after step 1 they are the first step's fields, as KineticSolverASub
  // exports them after AmbipolarEfieldSub, _8_0_0_1_KineticSolverA.f90:
  // 363-536); k_cell_moments copies the same values at later master steps
  for (int Q = threadIdx.x; Q < nq; Q += blockDim.x) {
    const int64_t g = T.coff + Q;
    c.mom[KAOS_EGMAG * c.ncell_total + g] = c.EG[g];
    if (a.have_import || !a.eamb) c.mom[KAOS_EAMAG * c.ncell_total + g] = c.EAmag[g];
  }
  if (a.have_import || !a.eamb) return;  // imported EAmag kept as is
  for (int Q = threadIdx.x; Q < nq; Q += blockDim.x) {
    M0f[Q] = a.momfilter ? filter_cell(M0p, nq, Q, a.fpM0) : M0p[Q];
    c.mom[KAOS_M0FILT * c.ncell_total + T.coff + Q] = M0f[Q];  // M0FiltAvrgRT
  }
  __syncthreads();
  const double S = T.sgn;  // qGL(1) <= 0 ? +1 : -1
  for (int Q = threadIdx.x; Q < nq; Q += blockDim.x) {
    const int64_t g = T.coff + Q;
    double ep = 0.0;
    if (M0p[Q] != 0.0 && a.eapressure) {
      const double *Mn = M0f;
      double R1 = (1.0 / fabs(c.hqC[g])) * (KB * c.Te[g] / (T.qs * Mn[Q]));
      double st, den;
      if (Q == 0) {
        st = -25.0 * Mn[Q] + 48.0 * Mn[Q + 1] - 36.0 * Mn[Q + 2] +
             16.0 * Mn[Q + 3] - 3.0 * Mn[Q + 4];
        den = 12.0 * c.dqC[g];
      } else if (Q == nq - 1) {
        st = -25.0 * Mn[Q] + 48.0 * Mn[Q - 1] - 36.0 * Mn[Q - 2] +
             16.0 * Mn[Q - 3] - 3.0 * Mn[Q - 4];
        den = -12.0 * c.dqC[g];
      } else if (Q == 1 || Q == nq - 2) {
        st = Mn[Q + 1] - Mn[Q - 1];
        den = 2.0 * c.dqC[g];
      } else {
        st = Mn[Q - 2] - 8.0 * Mn[Q - 1] + 8.0 * Mn[Q + 1] - Mn[Q + 2];
        den = 12.0 * c.dqC[g];
      }
      double R2 = a.eambsign ? -(st) / (-S * den) : fabs(st) / den;
      double R = R1 * R2;
      ep = a.eambsign ? R : fabs(R);
    }
    EP[Q] = ep;
  }
  __syncthreads();
  for (int Q = threadIdx.x; Q < nq; Q += blockDim.x) {
    double v = EP[Q];
    if (a.eambself && Q <= 2 && nq > 3 && M0p[Q] != 0.0 && a.eapressure) v = EP[3];
    c.EAmag[T.coff + Q] = 0.0 + v;  // EAInertial = 0 (EAINERTIALflag = 0)
    c.mom[KAOS_EAMAG * c.ncell_total + T.coff + Q] = 0.0 + v;
  }
}

// ---------------------------------------------------------------------------
// The one occupied bin of a marginal (all the cell's ions share it), or -1.
// A cell whose ions share one bin of an axis has that bin's centre as its
// first moment along the axis (the exact value of the ratio of sums), so the
// centred second-moment integrand of that bin is zero and falls back to the
// uncentred one (_8_6_6_SecondParIonMoment.f90:90-99) on every path.
__device__ __forceinline__ int warp_single_bin(const unsigned *m, int n) {
  int nz = 0, last = -1;
  for (int k = threadIdx.x & 31; k < n; k += 32)
    if (m[k]) { ++nz; last = k; }
  for (int o = 16; o > 0; o >>= 1) {
    nz += __shfl_xor_sync(0xffffffffu, nz, o);
    last = max(last, __shfl_xor_sync(0xffffffffu, last, o));
  }
  return nz == 1 ? last : -1;
}

__device__ __forceinline__ int single_bin(const unsigned *m, int n) {
  int nz = 0, last = -1;
  for (int k = 0; k < n; ++k)
    if (m[k]) { ++nz; last = k; }
  return nz == 1 ? last : -1;
}

// Moments of one cell from its count and binning marginals, for the
// allocation-free statistics entry point (ZerothIonMoment
// .. SecondParIonMoment _8_6_1-_8_6_6 with the NonUniform2D/3D integrators
// _8_5_*): every integrand there is a sum of single-axis terms at the bin
// centres, so the per-axis marginal counts carry all the information.
// M[] is indexed by the KAOS_M* selectors 0..9.
__device__ void cell_moments(double w, double cnt, const unsigned *mp,
                             const unsigned *m1, const unsigned *m2,
                             const double *epar, const double *e1,
                             const double *e2, int npar, int n1, int n2,
                             int three_d, int cenpar, int cenperp, double ms,
                             double M[10]) {
  for (int k = 0; k < 10; ++k) M[k] = 0.0;
  const double NqRT = cnt * w;
  double Nin = 0.0;
  for (int k = 0; k < npar; ++k) Nin += (double)mp[k];
  if (NqRT == 0.0 || Nin == 0.0) return;
  const double M0 = w * Nin;
  double Sp = 0.0, S1 = 0.0;
  for (int k = 0; k < npar; ++k) Sp += 0.5 * (epar[k] + epar[k + 1]) * mp[k];
  for (int k = 0; k < n1; ++k) S1 += 0.5 * (e1[k] + e1[k + 1]) * m1[k];
  const int kp = single_bin(mp, npar), k1 = single_bin(m1, n1);
  const double M1par = kp >= 0 ? 0.5 * (epar[kp] + epar[kp + 1]) : (w * Sp) / M0;
  double Tp = 0.0, Tq = 0.0, T1 = 0.0, T1c = 0.0;
  // centred integrand; for M2|| a bin whose centred value is exactly zero
  // falls back to the uncentred one (_8_6_6_SecondParIonMoment.f90:90-99).
  // The total-energy integrand also carries the Vperp terms, so it is never
  // zero and keeps the centred value (Tq).
  for (int k = 0; k < npar; ++k) {
    if (!mp[k]) continue;
    const double vc = 0.5 * (epar[k] + epar[k + 1]);
    const double d = cenpar ? (vc - M1par) : vc;
    double d2 = d * d;
    Tq += d2 * mp[k];
    if (d2 == 0.0) d2 = vc * vc;
    Tp += d2 * mp[k];
  }
  const double M1p1 = k1 >= 0 ? 0.5 * (e1[k1] + e1[k1 + 1]) : (w * S1) / M0;
  for (int k = 0; k < n1; ++k) {
    if (!m1[k]) continue;
    const double vc = 0.5 * (e1[k] + e1[k + 1]);
    T1 += vc * vc * m1[k];
    const double d = vc - M1p1;
    double d2 = d * d;
    if (d2 == 0.0) d2 = vc * vc;
    T1c += d2 * m1[k];
  }
  M[KAOS_M0] = M0;
  M[KAOS_M1PAR] = M1par;
  M[KAOS_M2PAR] = (ms / 2.0) * ((w * Tp) / M0);
  if (three_d) {
    double S2 = 0.0, T2 = 0.0, T2c = 0.0;
    for (int k = 0; k < n2; ++k) S2 += 0.5 * (e2[k] + e2[k + 1]) * m2[k];
    const int k2 = single_bin(m2, n2);
    const double M1p2 = k2 >= 0 ? 0.5 * (e2[k2] + e2[k2 + 1]) : (w * S2) / M0;
    for (int k = 0; k < n2; ++k) {
      if (!m2[k]) continue;
      const double vc = 0.5 * (e2[k] + e2[k + 1]);
      T2 += vc * vc * m2[k];
      const double d = vc - M1p2;
      double d2 = d * d;
      if (d2 == 0.0) d2 = vc * vc;
      T2c += d2 * m2[k];
    }
    M[KAOS_M1PERP1] = M1p1;
    M[KAOS_M1PERP2] = M1p2;
    M[KAOS_M2] = (ms / 2.0) * ((w * (T1 + T2 + Tq)) / M0);
    M[KAOS_M2PERP1] = (ms / 2.0) * ((w * (cenperp ? T1c : T1)) / M0);
    M[KAOS_M2PERP2] = (ms / 2.0) * ((w * (cenperp ? T2c : T2)) / M0);
  } else {
    M[KAOS_M1PERP] = M1p1;
    M[KAOS_M2] = (ms / 2.0) * ((w * (T1 + Tq)) / M0);
    M[KAOS_M2PERP] = (ms / 2.0) * ((w * (cenperp ? T1c : T1)) / M0);
  }
}

// ---------------------------------------------------------------------------
// Moments of one master step from the binning marginals (ZerothIonMoment ..
// SecondParIonMoment _8_6_1-_8_6_6 with the NonUniform2D/3D integrators
// _8_5_*): one warp per cell, lanes over the velocity bins.  Every
// integrand there is a sum of single-axis terms at the bin centres, so the
// per-axis marginal counts carry all the information.
__global__ void __launch_bounds__(256) k_cell_moments(TubeArgs a,
                                                      const int *cell_tube) {
  const int64_t g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const CellTables &c = a.ct;
  const int64_t NC = c.ncell_total;
  if (g >= NC) return;  // whole warp
  const TubeD &T = a.tubes[cell_tube[g]];
  const double ms = T.ms;
  const int n1 = c_vg.n1, n2 = c_vg.n2, npar = c_vg.npar;
  const double w = T.nsnormfac / c.d3xC[g];
  const double NqRT = (double)a.acc.cnt[g] * w;
  const unsigned *mp = a.acc.mpar + g * npar, *m1 = a.acc.m1 + g * n1;
  const unsigned *m2 = a.three_d ? a.acc.m2 + g * n2 : nullptr;
  double Nin = 0.0, Sp = 0.0, S1 = 0.0, S2 = 0.0;
  for (int k = lane; k < npar; k += 32) {
    const double m = (double)mp[k];
    Nin += m;
    Sp += 0.5 * (c_vg.epar[k] + c_vg.epar[k + 1]) * m;
  }
  for (int k = lane; k < n1; k += 32) S1 += 0.5 * (c_vg.e1[k] + c_vg.e1[k + 1]) * (double)m1[k];
  if (m2)
    for (int k = lane; k < n2; k += 32) S2 += 0.5 * (c_vg.e2[k] + c_vg.e2[k + 1]) * (double)m2[k];
  Nin = warp_sum(Nin);
  Sp = warp_sum(Sp);
  S1 = warp_sum(S1);
  S2 = warp_sum(S2);
  // the one occupied bin of each axis, or -1 (see warp_single_bin)
  const int kp = warp_single_bin(mp, npar), k1 = warp_single_bin(m1, n1);
  const int k2 = m2 ? warp_single_bin(m2, n2) : -1;
  double M[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (NqRT != 0.0 && Nin != 0.0) {
    const double M0 = w * Nin;
    const double M1par = kp >= 0 ? 0.5 * (c_vg.epar[kp] + c_vg.epar[kp + 1]) : (w * Sp) / M0;
    const double M1p1 = k1 >= 0 ? 0.5 * (c_vg.e1[k1] + c_vg.e1[k1 + 1]) : (w * S1) / M0;
    const double M1p2 = k2 >= 0 ? 0.5 * (c_vg.e2[k2] + c_vg.e2[k2 + 1]) : (w * S2) / M0;
    // centred integrand; for M2|| a bin whose centred value is exactly zero
    // falls back to the uncentred one (_8_6_6_SecondParIonMoment.f90:90-99).
    // The total-energy integrand also carries the Vperp terms, so it is
    // never zero and keeps the centred value (Tq).
    double Tp = 0.0, Tq = 0.0, T1 = 0.0, T1c = 0.0, T2 = 0.0, T2c = 0.0;
    for (int k = lane; k < npar; k += 32) {
      if (!mp[k]) continue;
      const double vc = 0.5 * (c_vg.epar[k] + c_vg.epar[k + 1]);
      const double d = a.cenpar ? (vc - M1par) : vc;
      double d2 = d * d;
      Tq += d2 * mp[k];
      if (d2 == 0.0) d2 = vc * vc;
      Tp += d2 * mp[k];
    }
    for (int k = lane; k < n1; k += 32) {
      if (!m1[k]) continue;
      const double vc = 0.5 * (c_vg.e1[k] + c_vg.e1[k + 1]);
      T1 += vc * vc * m1[k];
      const double d = vc - M1p1;
      double d2 = d * d;
      if (d2 == 0.0) d2 = vc * vc;
      T1c += d2 * m1[k];
    }
    if (m2)
      for (int k = lane; k < n2; k += 32) {
        if (!m2[k]) continue;
        const double vc = 0.5 * (c_vg.e2[k] + c_vg.e2[k + 1]);
        T2 += vc * vc * m2[k];
        const double d = vc - M1p2;
        double d2 = d * d;
        if (d2 == 0.0) d2 = vc * vc;
        T2c += d2 * m2[k];
      }
    Tp = warp_sum(Tp);
    Tq = warp_sum(Tq);
    T1 = warp_sum(T1);
    T1c = warp_sum(T1c);
    T2 = warp_sum(T2);
    T2c = warp_sum(T2c);
    M[KAOS_M0] = M0;
    M[KAOS_M1PAR] = M1par;
    M[KAOS_M2PAR] = (ms / 2.0) * ((w * Tp) / M0);
    if (a.three_d) {
      M[KAOS_M1PERP1] = M1p1;
      M[KAOS_M1PERP2] = M1p2;
      M[KAOS_M2] = (ms / 2.0) * ((w * (T1 + T2 + Tq)) / M0);
      M[KAOS_M2PERP1] = (ms / 2.0) * ((w * (a.cenperp ? T1c : T1)) / M0);
      M[KAOS_M2PERP2] = (ms / 2.0) * ((w * (a.cenperp ? T2c : T2)) / M0);
    } else {
      M[KAOS_M1PERP] = M1p1;
      M[KAOS_M2] = (ms / 2.0) * ((w * (T1 + Tq)) / M0);
      M[KAOS_M2PERP] = (ms / 2.0) * ((w * (a.cenperp ? T1c : T1)) / M0);
    }
  }
  if (lane == 0) {
    double *mom = c.mom;
    for (int k = 0; k < 10; ++k) mom[k * NC + g] = M[k];
    mom[KAOS_NQ * NC + g] = NqRT;
    c.M0prev[g] = M[KAOS_M0];
    mom[KAOS_EAMAG * NC + g] = c.EAmag[g];
    mom[KAOS_EGMAG * NC + g] = c.EG[g];
  }
}

// PoissonRNGSub (_3_2_PoissonRNG.f90:31-38): the number of uniforms whose
// running product stays above exp(-mean), the uniforms drawn from the
// Poisson stream keyed by (seed, cell Q, master step nn), two per Philox
// draw (at most 1e5 uniforms).  Also evaluated by the diagnostic sampler
// kaos_sample_rng.
__device__ __forceinline__ int64_t poisson_draw(uint64_t seed, uint32_t Q,
                                                uint32_t nn, double mean) {
  const double e = exp(-mean);
  double prod = 1.0;
  int64_t k = -1;
  uint32_t it = 0;
  while (prod > e && it < 100000u) {
    kaos_u32x4 w = kaos_philox(Q, nn, it >> 1, (KAOS_RNG_POIS << 24), seed);
    prod *= (it & 1u) ? kaos_u01(w.v[2], w.v[3]) : kaos_u01(w.v[0], w.v[1]);
    ++k;
    ++it;
  }
  return k;
}

// Model-A collision counts of one master step (IonNeutralCollision
// FrequencyASub _8_6_6_1_...:28-301) from the moments of k_cell_moments.
// One block per tube.
__global__ void k_collision_counts(TubeArgs a) {
  extern __shared__ double sm[];
  const TubeD T = a.tubes[blockIdx.x];
  const int nq = T.nq;
  const CellTables &c = a.ct;
  const int64_t NC = c.ncell_total;
  double *mom = c.mom;
  const uint32_t nn = a.dstep ? *a.dstep / (uint32_t)a.ndatfac + 1u : a.nn;
  double *f1p = sm, *f11 = sm + nq, *f12 = sm + 2 * nq, *f2p = sm + 3 * nq;
  double *s1p = sm + 4 * nq, *s11 = sm + 5 * nq, *s12 = sm + 6 * nq, *s2p = sm + 7 * nq;
  const int m1i = a.three_d ? KAOS_M1PERP1 : KAOS_M1PERP;
  for (int Q = threadIdx.x; Q < nq; Q += blockDim.x) {
    const int64_t g = T.coff + Q;
    s1p[Q] = mom[KAOS_M1PAR * NC + g];
    s11[Q] = mom[m1i * NC + g];
    s12[Q] = a.three_d ? mom[KAOS_M1PERP2 * NC + g] : 0.0;
    s2p[Q] = mom[KAOS_M2PAR * NC + g];
  }
  __syncthreads();
  for (int Q = threadIdx.x; Q < nq; Q += blockDim.x) {
    f1p[Q] = a.momfilter ? filter_cell(s1p, nq, Q, a.fpM1par) : s1p[Q];
    f11[Q] = a.momfilter ? filter_cell(s11, nq, Q, a.fpM1p1) : s11[Q];
    f12[Q] = a.momfilter ? filter_cell(s12, nq, Q, a.fpM1p2) : s12[Q];
    f2p[Q] = a.momfilter ? filter_cell(s2p, nq, Q, a.fpM2par) : s2p[Q];
  }
  __syncthreads();
  for (int Q = threadIdx.x; Q < nq; Q += blockDim.x) {
    const int64_t g = T.coff + Q;
    const double M0 = mom[KAOS_M0 * NC + g];
    double sigma = 0.0, nu = 0.0;
    if (M0 != 0.0 && f2p[Q] != 0.0) {
      double E = (6.242e18) * (1e-3) * f2p[Q];
      double l = 4.07 - 0.269 * log(E);
      sigma = (l * l) * pow(1.0 - exp(-415.0 / E), 0.8);
    }
    if (M0 != 0.0) {
      const uint64_t key = ((uint64_t)nn << 32) | (uint32_t)Q;
      double G0 = gauss64(a.seed, key, 0u, KAOS_RNG_NEUT, 0);
      double G1 = gauss64(a.seed, key, 0u, KAOS_RNG_NEUT, 1);
      double G2 = gauss64(a.seed, key, 0u, KAOS_RNG_NEUT, 2);
      double sN = sqrt(KB * a.TNeut / a.mNeut);
      double th = c.thetaGC[g], el = c.ellGC[g];
      double ct = cos(th), st = sin(th), sl = sqrt(el);
      double MVx = T.cphi * (3.0 * f1p[Q] * ct * st + f11[Q] * (1.0 - 3.0 * ct * ct)) / sl - f12[Q] * T.sphi;
      double MVy = T.sphi * (3.0 * f1p[Q] * ct * st + f11[Q] * (1.0 - 3.0 * ct * ct)) / sl + f12[Q] * T.cphi;
      double MVz = f1p[Q] * (3.0 * ct * ct - 1.0) / sl + 3.0 * f11[Q] * ct * st / sl;
      double dx = MVx - sN * G0, dy = MVy - sN * G1, dz = MVz - sN * G2;
      double vrel = sqrt(dx * dx + dy * dy + dz * dz);
      if (sigma != 0.0) {
        double mean = c.nsnormCNeut[g] * sigma * vrel * a.h;
        nu = (double)poisson_draw(a.seed, (uint32_t)Q, nn, mean);
        double cnt = (double)a.acc.cnt[g];
        if (nu > cnt) nu = cnt;
      }
    }
    c.nuPoi[g] = nu;
    mom[KAOS_NUPOI * NC + g] = nu;
  }
}

// ---------------------------------------------------------------------------
// Order-preserving removal (BCReIndexSub, Fortran pack, _8_0_7_1_BCReIndex
// .f90:33-131) in three passes: count kept per block, scan block counts per
// tube, scatter with in-block ranks.
struct Field {
  void *src, *dst;
  int size;
};
constexpr int MAXF = 14;
struct Fields {
  Field f[MAXF];
  int n;
};

struct BcArgs {
  const TubeD *tubes;
  const int *blk_tube;
  const int64_t *blk_start;
  const int *tube_blk0;  // first block of each tube (ntubes+1)
  int chunk;
  int64_t *nlive;
  const int32_t *qind;
  int64_t *blkcnt, *blkoff;
  unsigned long long *lb_out, *ub_out;  // per tube escape counts
  Fields fields;
  int ena;  // 1: operate on the ENA segments (tube.eoff) instead of ions
  // k_bc_mark: the slot arrays marked DEAD (x: mixed precision only)
  int32_t *qind_w;
  double *x_w;
};

__device__ __forceinline__ bool keep_slot(int q) {
  return q != BELOW && q != ABOVE && q != DEAD;
}

__global__ void k_bc_count(BcArgs a) {
  const int t = a.blk_tube[blockIdx.x];
  const TubeD &T = a.tubes[t];
  const int64_t toff = a.ena ? T.eoff : T.off;
  const int64_t nl = a.ena ? min(a.nlive[t], T.ecap) : a.nlive[t];
  const int64_t beg = a.blk_start[blockIdx.x];
  const int64_t end = min(beg + (int64_t)a.chunk, nl);
  int kept = 0, lb = 0, ub = 0;
  for (int64_t i = beg + threadIdx.x; i < end; i += blockDim.x) {
    int q = a.qind[toff + i];
    kept += keep_slot(q);
    lb += (q == BELOW);
    ub += (q == ABOVE);
  }
  for (int o = 16; o > 0; o >>= 1) {
    kept += __shfl_down_sync(0xffffffffu, kept, o);
    lb += __shfl_down_sync(0xffffffffu, lb, o);
    ub += __shfl_down_sync(0xffffffffu, ub, o);
  }
  __shared__ int sk[32], sl[32], su[32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { sk[w] = kept; sl[w] = lb; su[w] = ub; }
  __syncthreads();
  if (threadIdx.x == 0) {
    int K = 0, L = 0, U = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { K += sk[k]; L += sl[k]; U += su[k]; }
    a.blkcnt[blockIdx.x] = K;
    if (L) atomicAdd(a.lb_out + t, (unsigned long long)L);
    if (U) atomicAdd(a.ub_out + t, (unsigned long long)U);
  }
}

// Removal without moving the arrays: the escaped ions of a master step are
// counted and marked DEAD in place, as slots converted to ENAs are; the
// live ions keep their order, and a later compaction removes every DEAD
// slot at once.
__global__ void k_bc_mark(BcArgs a) {
  const int t = a.blk_tube[blockIdx.x];
  const TubeD &T = a.tubes[t];
  const int64_t nl = a.nlive[t];
  const int64_t beg = a.blk_start[blockIdx.x];
  const int64_t end = min(beg + (int64_t)a.chunk, nl);
  int lb = 0, ub = 0;
  // the indices of a tile of MARK_IT slots per thread are loaded before any
  // is examined, so their HBM latencies overlap
  constexpr int MARK_IT = 8;
  for (int64_t i0 = beg; i0 < end; i0 += (int64_t)MARK_IT * blockDim.x) {
    int q[MARK_IT];
#pragma unroll
    for (int k = 0; k < MARK_IT; ++k) {
      const int64_t i = i0 + k * (int64_t)blockDim.x + threadIdx.x;
      q[k] = i < end ? a.qind_w[T.off + i] : 0;
    }
#pragma unroll
    for (int k = 0; k < MARK_IT; ++k) {
      if (q[k] == BELOW || q[k] == ABOVE) {
        const int64_t j = T.off + i0 + k * (int64_t)blockDim.x + threadIdx.x;
        lb += (q[k] == BELOW);
        ub += (q[k] == ABOVE);
        a.qind_w[j] = DEAD;
        if (a.x_w) a.x_w[j] = XDEAD;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    lb += __shfl_down_sync(0xffffffffu, lb, o);
    ub += __shfl_down_sync(0xffffffffu, ub, o);
  }
  __shared__ int sl[32], su[32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { sl[w] = lb; su[w] = ub; }
  __syncthreads();
  if (threadIdx.x == 0) {
    int L = 0, U = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { L += sl[k]; U += su[k]; }
    if (L) atomicAdd(a.lb_out + t, (unsigned long long)L);
    if (U) atomicAdd(a.ub_out + t, (unsigned long long)U);
  }
}

// Exclusive scan of the kept counts over the blocks of one tube (one thread
// block per tube, block-wide scan in tiles), then the new live count.
__global__ void k_bc_scan(BcArgs a) {
  const int t = blockIdx.x;
  const int b0 = a.tube_blk0[t], b1 = a.tube_blk0[t + 1];
  __shared__ int64_t wsum[32];
  __shared__ int64_t base;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  const int l = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int r0 = b0; r0 < b1; r0 += blockDim.x) {
    const int b = r0 + threadIdx.x;
    const int64_t n = (b < b1) ? a.blkcnt[b] : 0;
    int64_t x = n;  // inclusive warp scan
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (l >= o) x += y;
    }
    if (l == 31) wsum[w] = x;
    __syncthreads();
    int64_t woff = 0, tot = 0;
    for (int v = 0; v < nw; ++v) { if (v < w) woff += wsum[v]; tot += wsum[v]; }
    if (b < b1) a.blkoff[b] = base + woff + x - n;
    __syncthreads();
    if (threadIdx.x == 0) base += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) a.nlive[t] = base;
}

__global__ void k_bc_scatter(BcArgs a, const int64_t *nlive_old) {
  const int t = a.blk_tube[blockIdx.x];
  const TubeD &T = a.tubes[t];
  const int64_t toff = a.ena ? T.eoff : T.off;
  const int64_t nl = a.ena ? min(nlive_old[t], T.ecap) : nlive_old[t];
  const int64_t beg = a.blk_start[blockIdx.x];
  const int64_t end = min(beg + (int64_t)a.chunk, nl);
  __shared__ int wsum[32];
  __shared__ int64_t base;
  if (threadIdx.x == 0) base = a.blkoff[blockIdx.x];
  __syncthreads();
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int64_t r0 = beg; r0 < end; r0 += blockDim.x) {
    const int64_t i = r0 + threadIdx.x;
    const bool in = i < end;
    const bool k = in && keep_slot(a.qind[toff + i]);
    const unsigned bal = __ballot_sync(0xffffffffu, k);
    const int wr = __popc(bal & ((1u << l) - 1u));
    if (l == 0) wsum[w] = __popc(bal);
    __syncthreads();
    int woff = 0, tot = 0;
    for (int q = 0; q < nw; ++q) { if (q < w) woff += wsum[q]; tot += wsum[q]; }
    if (k) {
      const int64_t src = toff + i, dst = toff + base + woff + wr;
      for (int f = 0; f < a.fields.n; ++f) {
        const Field &F = a.fields.f[f];
        if (F.size == 16)
          ((uint4 *)F.dst)[dst] = ((const uint4 *)F.src)[src];
        else if (F.size == 8)
          ((uint64_t *)F.dst)[dst] = ((const uint64_t *)F.src)[src];
        else
          ((uint32_t *)F.dst)[dst] = ((const uint32_t *)F.src)[src];
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) base += tot;
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Lower / upper boundary injection on a master step (BoundaryConditionsSub
// :743-809, KineticSolverBSub _8_0_0_2_KineticSolverB.f90:195-793,
// MBVelocityDistributionSub _6_1_MBVelocityDistribution.f90:29-120).
struct InjArgs {
  const TubeD *tubes;
  CellTables ct;
  Accum acc;
  Ions ion;
  int64_t *nlive;
  uint64_t *next_id;
  unsigned long long *n_in;  // per tube injected count (LB, UB)
  int mixed, ub, bin, exporting;
  int flux, stat;  // FLUXINJECTIONflag, STATICINJECTIONflag
  double ms, qs;
  uint64_t seed;
  uint32_t *status;
  unsigned *cxc;             // charge exchange on: selection-chunk counts
  const int *tube_cx0;
  int cx_stride, cx_chunk;
};

// Ions injected by one tube at this master step (capacity-clamped).
__device__ __forceinline__ int64_t inject_count(const InjArgs &a, const TubeD &T,
                                                int64_t nl) {
  const int64_t k = (int64_t)llrint(a.ub ? T.nsnormCUB : T.nsnormCLB);
  if (k <= 0) return 0;
  return nl + k > T.cap ? max(T.cap - nl, (int64_t)0) : k;
}

// grid (blocks per tube, tubes): every block of a tube reads the same live
// count; k_inject_commit advances it afterwards
__global__ void k_inject(InjArgs a) {
  const int t = blockIdx.y;
  const TubeD T = a.tubes[t];
  const int Q = a.ub ? T.nq - 1 : 0;
  const int64_t g = T.coff + Q;
  const int64_t nl = a.nlive[t];
  const int64_t k = inject_count(a, T, nl);
  if (k <= 0) return;
  const double rho0 = a.ub ? T.rhoUB : T.rhoLB, z0 = a.ub ? T.zUB : T.zLB;
  const double r = sqrt(rho0 * rho0 + z0 * z0);
  const double ct = z0 / r, st = rho0 / r, el = 1.0 + 3.0 * ct * ct, sl = sqrt(el);
  const double sig = sqrt(KB * a.ct.TsG[g] / T.ms);
  const double qm = T.qs / T.ms;
  const double aea = fabs(qm * fabs(a.ct.EAmag[g])), ag = fabs(qm * fabs(a.ct.EG[g]));
  const double qc = a.ct.qGC[g];
  const uint64_t id0 = a.next_id[t];
  const bool d3 = c_vg.three_d;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < k;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = T.off + nl + i;
    const uint64_t id = id0 + (uint64_t)i;
    const double Vx0 = sig * gauss64(a.seed, id, 0u, KAOS_RNG_INJECT, 0);
    const double Vy0 = sig * gauss64(a.seed, id, 0u, KAOS_RNG_INJECT, 1);
    const double Vz0 = sig * gauss64(a.seed, id, 0u, KAOS_RNG_INJECT, 2);
    const double h_ = Vx0 * T.cphi + Vy0 * T.sphi;
    double v1 = ((1.0 - 3.0 * ct * ct) / sl) * h_ + ((3.0 * Vz0 * ct * st) / sl);
    double vpar = ((3.0 * ct * st) / sl) * h_ + ((Vz0 * (3.0 * ct * ct - 1.0)) / sl);
    double v2 = -Vx0 * T.sphi + Vy0 * T.cphi;
    if (a.flux) {  // V|| of the Maxwellian flux into the tube (Rayleigh)
      kaos_u32x4 w = kaos_philox((uint32_t)id, (uint32_t)(id >> 32), 0u,
                                 (KAOS_RNG_INJECT << 24) | 3u, a.seed);
      const double r = sig * sqrt(-2.0 * log(kaos_u01(w.v[0], w.v[1])));
      vpar = a.ub ? -r : r;
    }
    if (a.stat) v1 = v2 = vpar = 0.0;  // STATICINJECTIONflag
    const double vp = vperp_mag(v1, v2);
    int bp = vbin(c_vg.epar, c_vg.npar, vpar);
    int b1 = vbin(c_vg.e1, c_vg.n1, d3 ? v1 : vp);
    int b2 = d3 ? vbin(c_vg.e2, c_vg.n2, v2) : 0;
    if (a.ion.vb) a.ion.vb[j] = ((b1 + 1) << 16) | (bp + 1);
    if (a.mixed) {
      a.ion.x[j] = (double)Q + (qc - a.ct.qGL[g]) / (a.ct.qGH[g] - a.ct.qGL[g]);
      a.ion.vpar[j] = vpar;
      a.ion.v12[j] = make_double2(v1, v2);
      a.ion.ffl[j] = make_float2((float)aea, (float)ag);
      a.ion.fqk4[j] = (float)qc;
    } else {
      a.ion.rho[j] = rho0;
      a.ion.z[j] = z0;
      a.ion.vpar[j] = vpar;
      a.ion.v1[j] = v1;
      a.ion.v2[j] = v2;
      a.ion.aea[j] = aea;
      a.ion.ag[j] = ag;
      a.ion.qk4[j] = qc;
      if (a.ion.rho4) {  // k4 point before the first push: where it stands
        a.ion.rho4[j] = rho0;
        a.ion.z4[j] = z0;
      }
    }
    a.ion.qind[j] = Q;
    a.ion.id[j] = id;
    if (a.cxc)
      agg_inc(a.cxc, (int64_t)(a.tube_cx0[t] + (int)((nl + i) / a.cx_chunk)) * a.cx_stride + Q);
    if (a.bin) accumulate(a.acc, T, Q, b1, d3 ? b2 : 0, bp, a.exporting);
  }
}

// After k_inject: advance the live counts and ids (one thread per tube) and
// flag a capacity clamp.
__global__ void k_inject_commit(InjArgs a, int ntubes) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntubes) return;
  const TubeD &T = a.tubes[t];
  const int64_t nl = a.nlive[t];
  const int64_t want = (int64_t)llrint(a.ub ? T.nsnormCUB : T.nsnormCLB);
  const int64_t k = inject_count(a, T, nl);
  if (want > 0 && k < want) atomicOr(a.status, ST_CAP);
  a.nlive[t] = nl + k;
  a.next_id[t] += (uint64_t)k;
  a.n_in[t] = (unsigned long long)k;
}

// ---------------------------------------------------------------------------
// Initial ions on the device (kaos_init_particles): the draws of the CPU
// oracle's generator (orc_init), then the derived per-ion state that
// kaos_load_particles computes on the host.  Products and sums of the draws
// are written with explicit rounding so that no multiply-add is fused.
struct InitArgs {
  TubeD T;
  const int64_t *pre;   // [nq+1] exclusive prefix of the per-cell counts
  int64_t n;
  uint64_t id0;         // id of ion 0 (keys its draws)
  Ions ion;
  CellTables ct;
  double tail_fraction, s_tail;
  int nu;               // Student-t degrees of freedom of the kappa tail
  uint64_t seed;
  int mixed;
};

// One new ion j of tube T in cell c at q with field-aligned velocity: the
// per-ion state every path starts from (Qindk1, id, 2D bins; mixed: the
// cell coordinate and the velocities; FP64: meridian-plane position from the
// quartic root by Newton from the cell's linear guess, converged to FP64).
__device__ __forceinline__ void store_ion(const Ions &I, const TubeD &T,
                                          const CellTables &ct, int64_t j,
                                          uint64_t id, int c, double q,
                                          double vpar, double v1, double v2,
                                          int mixed) {
  const int64_t k = T.off + j, g = T.coff + c;
  const double qL = ct.qGL[g], qH = ct.qGH[g];
  I.qind[k] = c;
  I.id[k] = id;
  if (I.vb) {
    const int bp = vbin(c_vg.epar, c_vg.npar, vpar);
    const int b1 = vbin(c_vg.e1, c_vg.n1, vperp_mag(v1, v2));
    I.vb[k] = ((b1 + 1) << 16) | (bp + 1);
  }
  if (mixed) {
    I.x[k] = (double)c + (q - qL) / (qH - qL);
    I.vpar[k] = vpar;
    I.v12[k] = make_double2(v1, v2);
    I.fqk4[k] = (float)q;
  } else {
    const double fr = (q - qL) / (qH - qL);
    const double u0 = ct.uL[g] + fr * (ct.uH[g] - ct.uL[g]);
    const double u = quartic_newton(q, 1.0 / T.pG, u0, 6);
    const double st = sqrt(u / T.pG), ctv = q * u * u, r = u * RE;
    double rho = r * st, z = r * ctv;
    if (fabs(rho) < 1e-6) rho = 0.0;
    if (fabs(z) < 1e-6) z = 0.0;
    I.rho[k] = rho;
    I.z[k] = z;
    I.vpar[k] = vpar;
    I.v1[k] = v1;
    I.v2[k] = v2;
    I.qk4[k] = q;
    // the k4 point of an ion not yet pushed is where it stands (charge
    // exchange may convert an injected ion before its first push)
    if (I.rho4) {
      I.rho4[k] = rho;
      I.z4[k] = z;
    }
  }
}

__device__ __forceinline__ void init_pair(uint64_t seed, uint64_t id,
                                          uint32_t sub, double &a, double &b) {
  kaos_u32x4 w = kaos_philox((uint32_t)id, (uint32_t)(id >> 32), 0u,
                             (KAOS_RNG_INIT << 24) | sub, seed);
  const double u1 = kaos_u01(w.v[0], w.v[1]), u2 = kaos_u01(w.v[2], w.v[3]);
  const double R = sqrt(__dmul_rn(-2.0, log(u1)));
  double sn, cs;
  sincos(__dmul_rn(__dmul_rn(2.0, PI), u2), &sn, &cs);
  a = __dmul_rn(R, cs);
  b = __dmul_rn(R, sn);
}

__global__ void k_init(InitArgs a) {
  const TubeD &T = a.T;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < a.n;
       j += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = T.nq;  // cell: pre[lo] <= j < pre[lo + 1]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (a.pre[mid] <= j) lo = mid; else hi = mid;
    }
    const int c = lo;
    const int64_t g = T.coff + c;
    const double qL = a.ct.qGL[g], qH = a.ct.qGH[g];
    const uint64_t id = a.id0 + (uint64_t)j;
    kaos_u32x4 w = kaos_philox((uint32_t)id, (uint32_t)(id >> 32), 0u,
                               (KAOS_RNG_INIT << 24), a.seed);
    const double upos = kaos_u01(w.v[0], w.v[1]), upop = kaos_u01(w.v[2], w.v[3]);
    const double q = __dadd_rn(qL, __dmul_rn(__dadd_rn(0.02, __dmul_rn(0.96, upos)),
                                             __dadd_rn(qH, -qL)));
    const bool tail = upop < a.tail_fraction;
    double g0, g1, g2, g3;
    init_pair(a.seed, id, 1u, g0, g1);
    init_pair(a.seed, id, 2u, g2, g3);
    double f;
    if (!tail) {
      f = sqrt(KB * a.ct.TsG[g] / T.ms);
    } else {
      double W = __dmul_rn(g3, g3), x, y;
      int m = 1;  // normals 3 .. 3+nu-1; g3 is the first
      for (uint32_t sub = 3; m < a.nu; ++sub) {
        init_pair(a.seed, id, sub, x, y);
        W = __dadd_rn(W, __dmul_rn(x, x));
        if (++m < a.nu) { W = __dadd_rn(W, __dmul_rn(y, y)); ++m; }
      }
      f = a.s_tail / sqrt(W / (double)a.nu);
    }
    const double vpar = __dmul_rn(f, g0), v1 = __dmul_rn(f, g1), v2 = __dmul_rn(f, g2);
    store_ion(a.ion, T, a.ct, j, id, c, q, vpar, v1, v2, a.mixed);
  }
}

// ---------------------------------------------------------------------------
// kaos_load_particles on the device: the KineticSolverASub q clamp
// (_8_0_0_1_KineticSolverA.f90:55-65), the cell of each ion and its derived
// state, from the caller's (q, V||, Vperp1, Vperp2) copied to the device.
struct LoadArgs {
  TubeD T;
  const double *q, *vpar, *v1, *v2;  // v2 may be null (2D grid)
  int64_t n;
  uint64_t id0;
  Ions ion;
  CellTables ct;
  int mixed;
};

__global__ void k_load(LoadArgs a) {
  extern __shared__ double E[];  // oriented cell edges [nq + 1]
  const TubeD &T = a.T;
  const double *qGL = a.ct.qGL + T.coff, *qGH = a.ct.qGH + T.coff;
  for (int k = threadIdx.x; k <= T.nq; k += blockDim.x)
    E[k] = (k < T.nq) ? T.sgn * qGL[k] : T.sgn * qGH[T.nq - 1];
  __syncthreads();
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < a.n;
       j += (int64_t)gridDim.x * blockDim.x) {
    double q = a.q[j];
    const double s = T.sgn * q;
    if (s <= E[0]) q = qGL[0];
    else if (s > E[T.nq]) q = qGH[T.nq - 1];
    const int c = cell_search(E, T.nq, T.sgn * q);
    store_ion(a.ion, T, a.ct, j, a.id0 + (uint64_t)j, c, q, a.vpar[j], a.v1[j],
              a.v2 ? a.v2[j] : 0.0,
              a.mixed);
  }
}

// ---------------------------------------------------------------------------
// ConvectionSub (_8_11_Convection.f90:135-258): on a master step the tube's
// field line moves to L-shell p_new (the E x B drift); every ion keeps its q
// and its V||, is placed on the new field line (RK4DipolePolynomialSolverSub
// at (q, p_new)), and its magnetic moment mu = m Vperp^2 / (2 B) is kept, so
// both Vperp components (same gyro-angle) scale by sqrt(B_new / B_old).
// Runs with the tube's old tables, before the new ones are copied in.
struct ConvArgs {
  TubeD T;               // the tube before the move
  double p_new;
  const int64_t *nlive;
  int tube;
  Ions ion;
  CellTables ct;
  int mixed;
};

// |B| / B0 at (q, u = r/RE) on any field line: sqrt(1 + 3 cos^2) / u^3.
__device__ __forceinline__ double bnorm(double q, double u) {
  const double ct = q * u * u;
  return sqrt(1.0 + 3.0 * ct * ct) / (u * u * u);
}

// The queued moves of one master step in one launch: blockIdx.y = the move
// (its entry and new L-shell), blockIdx.x strides over the entry's ions.
struct ConvManyArgs {
  const TubeD *tubes;   // the descriptors before the moves
  const int *tube;      // per move: the entry
  const double *p_new;  // per move: the new L-shell
  const int64_t *nlive;
  Ions ion;
  CellTables ct;
  int mixed;
};

__device__ __forceinline__ void convect_ions(const ConvArgs &a) {
  const TubeD &T = a.T;
  const int64_t nl = a.nlive[a.tube];
  const double ip_old = 1.0 / T.pG, ip_new = 1.0 / a.p_new;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  // the next ion's Qindk1 and position are loaded before the current ion is
  // moved, so their memory latency overlaps its Newton solves
  int n_qi = DEAD;
  double n_a = 0.0, n_b = 0.0;
  if (i < nl) {
    const int64_t j = T.off + i;
    n_qi = a.ion.qind[j];
    if (a.mixed) n_a = a.ion.x[j];
    else { n_a = a.ion.rho[j]; n_b = a.ion.z[j]; }
  }
  for (; i < nl; i += stride) {
    const int64_t j = T.off + i;
    const int qd = n_qi;
    const double pa = n_a, pb = n_b;
    if (i + stride < nl) {
      const int64_t jn = j + stride;
      n_qi = a.ion.qind[jn];
      if (a.mixed) n_a = a.ion.x[jn];
      else { n_a = a.ion.rho[jn]; n_b = a.ion.z[jn]; }
    }
    if (qd == DEAD) continue;
    double q, u_old;
    if (a.mixed) {
      const double x = pa;
      if (x < XDEAD_LIM) continue;
      const int c = x_cell(x, T.nq);
      const int64_t g = T.coff + c;
      const double o = x - (double)c;
      q = a.ct.qGL[g] + o * (a.ct.qGH[g] - a.ct.qGL[g]);
      u_old = quartic_newton_conv(q, ip_old, a.ct.uL[g] + o * (a.ct.uH[g] - a.ct.uL[g]), 8);
    } else {
      const double rho = pa, z = pb;
      const double r2 = rho * rho + z * z, r = sqrt(r2);
      q = (RE * RE) * (z / r) / r2;
      u_old = r / RE;
    }
    const double u_new = quartic_newton_conv(q, ip_new, u_old, 8);
    const double f = sqrt(bnorm(q, u_new) / bnorm(q, u_old));
    if (a.mixed) {
      const double2 v = a.ion.v12[j];
      a.ion.v12[j] = make_double2(f * v.x, f * v.y);
    } else {
      const double rr = u_new * RE, st = sqrt(u_new * ip_new), ctv = q * u_new * u_new;
      double rho = rr * st, z = rr * ctv;
      if (fabs(rho) < 1e-6) rho = 0.0;
      if (fabs(z) < 1e-6) z = 0.0;
      a.ion.rho[j] = rho;
      a.ion.z[j] = z;
      a.ion.v1[j] = f * a.ion.v1[j];
      a.ion.v2[j] = f * a.ion.v2[j];
    }
  }
}

__global__ void k_convect_many(ConvManyArgs m) {
  ConvArgs a;
  a.tube = m.tube[blockIdx.y];
  a.T = m.tubes[a.tube];
  a.p_new = m.p_new[blockIdx.y];
  a.nlive = m.nlive;
  a.ion = m.ion;
  a.ct = m.ct;
  a.mixed = m.mixed;
  convect_ions(a);
}

// The new per-cell tables and descriptors of the moved entries, from one
// staging copy: blockIdx.y = the move, blockIdx.x = the table.
constexpr int CONV_NTAB = 28;
struct TableApplyArgs {
  double *dst[CONV_NTAB];  // the per-cell tables (concatenated over entries)
  const double *stage;     // [move][table][nqmax]
  const TubeD *td;         // per move: the new descriptor
  const int *tube;         // per move: the entry
  TubeD *tubes;
  int nqmax;
};

__global__ void k_apply_tables(TableApplyArgs a) {
  const int p = blockIdx.y, k = blockIdx.x;
  const TubeD &T = a.td[p];
  const double *src = a.stage + ((int64_t)p * CONV_NTAB + k) * a.nqmax;
  for (int i = threadIdx.x; i < T.nq; i += blockDim.x) a.dst[k][T.coff + i] = src[i];
  if (k == 0 && threadIdx.x == 0) a.tubes[a.tube[p]] = T;
}

}  // namespace kaos

namespace kaos {

// ---------------------------------------------------------------------------
// kaos_get_particles on the device: field-line q in FP64 from the stored
// position (mixed: the cell coordinate; FP64: the meridian-plane point), the
// FP64 velocities and Qindk1, for the live ions only (slots
// converted to ENAs are skipped) in particle order.  Three passes: live
// count per block, exclusive scan of the block counts, in-order write.
constexpr int EXP_THREADS = 256, EXP_ITEMS = 8;  // 2048 ions per block

struct ExportArgs {
  Ions ion;
  int64_t off, nl;           // the tube's segment and live slots
  const double *qGL, *qGH;   // the tube's cell edges (mixed)
  int nq;                    // the tube's cells (mixed)
  int mixed, nb;
  unsigned *blkcnt;
  unsigned long long *blkoff, *total;
  double *q, *vpar, *v1, *v2;
  int32_t *qind;
};

__global__ void __launch_bounds__(EXP_THREADS) k_exp_count(ExportArgs a) {
  const int64_t beg = (int64_t)blockIdx.x * EXP_THREADS * EXP_ITEMS;
  unsigned n = 0;
  for (int k = 0; k < EXP_ITEMS; ++k) {
    const int64_t i = beg + k * EXP_THREADS + threadIdx.x;
    if (i < a.nl && a.ion.qind[a.off + i] != DEAD) ++n;
  }
  __shared__ unsigned ws[EXP_THREADS / 32];
  for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = n;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned t = 0;
    for (int w = 0; w < EXP_THREADS / 32; ++w) t += ws[w];
    a.blkcnt[blockIdx.x] = t;
  }
}

// exclusive scan of the block counts (one block of 1024 threads)
__global__ void __launch_bounds__(1024) k_exp_scan(ExportArgs a) {
  __shared__ unsigned long long ws[32], base;
  const int l = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  for (int r0 = 0; r0 < a.nb; r0 += blockDim.x) {
    const int b = r0 + threadIdx.x;
    const unsigned long long n = b < a.nb ? a.blkcnt[b] : 0ull;
    unsigned long long x = n;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (l >= o) x += y;
    }
    if (l == 31) ws[w] = x;
    __syncthreads();
    unsigned long long woff = 0, tot = 0;
    for (int v = 0; v < nw; ++v) { if (v < w) woff += ws[v]; tot += ws[v]; }
    if (b < a.nb) a.blkoff[b] = base + woff + x - n;
    __syncthreads();
    if (threadIdx.x == 0) base += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) *a.total = base;
}

__global__ void __launch_bounds__(EXP_THREADS) k_exp_write(ExportArgs a) {
  const int64_t beg = (int64_t)blockIdx.x * EXP_THREADS * EXP_ITEMS;
  __shared__ unsigned ws[EXP_THREADS / 32];
  const int l = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned long long done = a.blkoff[blockIdx.x];
  for (int k = 0; k < EXP_ITEMS; ++k) {
    const int64_t i = beg + k * EXP_THREADS + threadIdx.x;
    const int64_t j = a.off + i;
    int qi = DEAD;
    if (i < a.nl) qi = a.ion.qind[j];
    const bool live = qi != DEAD;
    const unsigned bal = __ballot_sync(0xffffffffu, live);
    if (l == 0) ws[w] = __popc(bal);
    __syncthreads();
    unsigned woff = 0, tot = 0;
    for (int v = 0; v < EXP_THREADS / 32; ++v) { if (v < w) woff += ws[v]; tot += ws[v]; }
    __syncthreads();  // ws is rewritten by the next tile
    if (live) {
      const int64_t o = (int64_t)(done + woff + __popc(bal & ((1u << l) - 1u)));
      double q, vp, v1, v2;
      if (a.mixed) {
        const double x = a.ion.x[j];
        const int c = x_cell(x, a.nq);
        q = fma(x - (double)c, a.qGH[c] - a.qGL[c], a.qGL[c]);
        vp = a.ion.vpar[j];
        const double2 v = a.ion.v12[j];
        v1 = v.x;
        v2 = v.y;
      } else {
        const double rho = a.ion.rho[j], z = a.ion.z[j];
        const double r2 = rho * rho + z * z, r = sqrt(r2);
        q = (RE * RE) * (z / r) / r2;
        vp = a.ion.vpar[j];
        v1 = a.ion.v1[j];
        v2 = a.ion.v2[j];
      }
      if (a.q) a.q[o] = q;
      if (a.vpar) a.vpar[o] = vp;
      if (a.v1) a.v1[o] = v1;
      if (a.v2) a.v2[o] = v2;
      if (a.qind) a.qind[o] = qi;
    }
    done += tot;
  }
}

}  // namespace kaos
