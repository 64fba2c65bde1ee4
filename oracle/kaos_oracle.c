/*
 * kaos_oracle.c -- CPU FP64 restatement of the KAOS per-timestep kinetic
 * particle loop for ONE flux tube.  TEST INFRASTRUCTURE ONLY: this file is
 * the checker for the CUDA path; only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load it.  Nothing in the product links it.
 *
 * Parity status: the reference (Fortran 90 + MPI) cannot be compiled in this
 * environment (no gfortran / mpif90) and ships no tests, fixtures or
 * recorded outputs.  This restatement is therefore pinned by analytic
 * known-answer tests and by the reference's own inline invariant checks
 * (quartic residual, p consistency, particle-number conservation,
 * F*d3v = N, moment/integrand consistency) -- "parity unpinned" against
 * reference outputs.
 *
 * It follows the reference routine by routine (file:line cited at each
 * function) in the reference's Cartesian formulation, including its quirks:
 * three force evaluations with k3 = k2, velocity rebuilt from V|| only,
 * per-step quartic re-projection with the complex resolvent-cubic formula,
 * lagged per-particle field magnitudes, start-of-step binning indices,
 * one-step-lagged escape detection and order-preserving compaction.
 *
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off -fno-fast-math).
 */
#ifndef ORC_OPS_COUNTED
#include <complex.h>
#endif
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../include/kaos_gpu.h"
#include "../include/kaos_philox.h"

/* Hooks of the op-counting build (oracle/op_count.cpp, which includes this
 * file with `double` replaced by a counting type).  In this plain C build
 * they do nothing and the complex arithmetic is C99's. */
#ifndef ORC_OPS_COUNTED
typedef double complex orc_cplx;
#define ORC_I I
#define orc_cacos cacos
#define orc_ccos ccos
#define orc_creal creal
#define ORC_PHASE(ph) ((void)0)
#define ORC_SEARCH_BEGIN() ((void)0)
#define ORC_SEARCH_END() ((void)0)
#endif
/* op-counting phases of one step */
#define ORC_PH_PUSH_ION 0
#define ORC_PH_PUSH_ENA 1
#define ORC_PH_CX 2
#define ORC_PH_MASTER 3

/* ---- _ModelInput.f90:35-43 physical constants ---------------------------- */
#define PI 3.14159265358979323846 /* a parameter: folded into constants */
#define KB 138e-25
#define EPS0 8.854e-12
#define MDIP 8.06e15
#define GG 667e-13
#define ME 598e22
#define RE 638e4

typedef struct orc {
  kaos_params_c P;
  /* tube */
  int nq;
  double pG, phiG, nsnormfac, nsnormCLB, nsnormCUB, sumdsICR;
  double *qGL, *qGH, *qGC, *hqC, *dqC, *d3xC, *rGC, *thetaGC, *ellGC, *TeG,
      *TsG, *nsnormCNeut, *lambdaPerp, *EtaLH, *XiPerp1, *XiPerp2, *S0,
      *OmegaG0, *ChiPerp1, *ChiPerp2;
  /* velocity grid */
  int n1, n2, npar, nv;
  double *e1, *e2, *epar, *c1, *c2, *cpar, *d3v;
  /* ENA velocity grid V3CellT (Vp, Vq, Vphi edges) */
  int nep, neq, neph;
  double *eep, *eeq, *eeph;
  /* particles */
  int64_t cap, np;
  double *x, *y, *z, *Vx, *Vy, *Vz, *V1, *V2, *Vp, *AEA, *AG, *AEAN, *AGN;
  double *qk4, *rk4, *thk4, *phk4, *ellk4, *Vpe, *Vphe; /* Vpe/Vphe: ENA Vp, Vphi */
  int64_t *Qind, *ipar, *i1, *i2;
  int64_t *iep, *ieq, *ieph; /* ENA Vpindk1, Vqindk1, Vphiindk1 (0: none) */
  unsigned char *ena;
  uint64_t *id;
  uint64_t next_id;
  /* per-cell state */
  double *Te, *EAmag, *EG, *M0prev, *nuPoi;
  double *mom[KAOS_NMOMENTS];
  int64_t *cnt, *hist;
  int have_import, export_on, literal, loaded;
  double *EAimport;
  int64_t n; /* computational steps taken */
  int64_t lb_out, ub_out, lb_in, ub_in;
  int64_t lbe_out, ube_out; /* escaped ENAs of the latest master step */
  kaos_tube_c *pending; /* orc_update_tube: applied at the next master step */
  double GAconv;        /* gyro-angle carried between ions as in the reference */
  char err[256];
} orc;

static void free_tube(kaos_tube_c *c);

/* ------------------------------------------------------------------------ */
/* helpers from _KineticMainParams.f90:568-815                              */
static double sq(double a) { return a * a; }

/* LinInterpsub _KineticMainParams.f90:810-815 */
static double lin_interp(double x, double y1, double y2, double x1, double x2) {
  return y1 + (((x - x1) / (x2 - x1)) * (y2 - y1));
}

static double *dup(const double *s, int n) {
  double *d = (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  if (s)
    memcpy(d, s, sizeof(double) * (size_t)n);
  return d;
}

/* hemisphere orientation: +1 when q increases from the lower boundary
 * (reference "qGLGT(nn,1) <= 0" branches), -1 otherwise.  All cell
 * searches and interpolations are written in the oriented coordinate
 * s = sgn*q, in which both reference branches are the same code. */
static double orient(const orc *o) { return o->qGL[0] <= 0.0 ? 1.0 : -1.0; }

/* Cell search, KineticUpdateA _8_1_1_KineticUpdateA.f90:221-273: first cell
 * is [lo,hi], later cells (lo,hi]; 0 below LB, -1 above UB (1-based).  */
static int64_t cell_search(const orc *o, double q) {
  ORC_SEARCH_BEGIN(); /* the orientation products stand for branches */
  double s = orient(o);
  double sq_ = s * q;
  int64_t idx = -9; /* "unset": the reference leaves Qindk1 unchanged */
  for (int k = 0; k < o->nq; ++k) {
    double lo = s * o->qGL[k], hi = s * o->qGH[k];
    if (k == 0) {
      if (lo <= sq_ && sq_ <= hi) {
        idx = 1;
        break;
      }
    } else if (lo < sq_ && sq_ <= hi) {
      idx = k + 1;
      break;
    }
  }
  if (s * o->qGL[0] > sq_)
    idx = 0;
  else if (s * o->qGH[o->nq - 1] < sq_)
    idx = -1;
  ORC_SEARCH_END();
  return idx;
}

/* Velocity-bin search, _8_1_1_KineticUpdateA.f90:994-1129.  3D grid:
 * out of range -> 0.  2D grid: no out-of-range branch, the index keeps its
 * previous value (`prev`). */
static int64_t vbin(const double *e, int n, double v, int oor_zero,
                    int64_t prev) {
  for (int k = 0; k < n; ++k) {
    if (oor_zero && ((e[0] > v) || (v > e[n])))
      return 0;
    if (k == 0) {
      if (e[0] <= v && v <= e[1])
        return 1;
    } else if (e[k] < v && v <= e[k + 1])
      return k + 1;
  }
  return prev;
}

/* ------------------------------------------------------------------------ */
/* RK4DipolePolynomialSolverSub _8_1_4_RK4DipolePolynomialSolver.f90:26-134:
 * quartic u^4 + u/(p q^2) - 1/q^2 = 0 through the resolvent cubic with
 * complex acos/cos, then (r, theta) and Cartesian (x, y, z). */
static void quartic(double qN, double pN, double phiN, double *r, double *th,
                    double *xf, double *yf, double *zf) {
  double Ap = 0.0, Bp = 0.0;
  double Cp = 1.0 / (pN * (qN * qN));
  double Dp = -1.0 / (qN * qN);
  double Ab = -Bp;
  double Bb = Ap * Cp - 4.0 * Dp;
  double Cb = 4.0 * Bp * Dp - Cp * Cp - (Ap * Ap) * Dp;
  double Abb = Bb - (Ab * Ab) / 3.0;
  double Bbb = 2.0 * (Ab * Ab * Ab) / 27.0 - Ab * Bb / 3.0 + Cb;
  double Delta = -Bbb / 2.0;
  double Eps = Abb / 3.0;
  orc_cplx I1 = ORC_I;
  orc_cplx Thetap = orc_cacos(Delta / (I1 * sqrt(Eps * Eps * Eps)));
  orc_cplx s23 =
      2.0 * I1 * sqrt(Eps) * orc_ccos((Thetap + 4.0 * PI) / 3.0) - Ab / 3.0;
  double sigma = fabs(orc_creal(s23));
  double mu = sqrt((Ap * Ap) / 4.0 - Bp + sigma);
  double pii;
  if (mu != 0.0)
    pii = sqrt(3.0 * (Ap * Ap) / 4.0 - (mu * mu) - 2.0 * Bp -
               (4.0 * Ap * Bp - 8.0 * Cp - (Ap * Ap * Ap)) / (4.0 * mu));
  else
    pii = sqrt(3.0 * (Ap * Ap) / 4.0 - 2.0 * Bp -
               2.0 * sqrt((sigma * sigma) - 4.0 * Dp));
  double gamma3 = -Ap / 4.0 - mu / 2.0 + pii / 2.0;
  double r3 = gamma3 * RE;
  double th3 = asin(sqrt(r3 / (RE * pN)));
  double thf = (qN <= 0.0) ? PI - th3 : th3;
  double x = r3 * sin(thf) * cos(phiN);
  double y = r3 * sin(thf) * sin(phiN);
  double z = r3 * cos(thf);
  if (fabs(x) < 1e-6)
    x = 0.0;
  if (fabs(y) < 1e-6)
    y = 0.0;
  if (fabs(z) < 1e-6)
    z = 0.0;
  *r = r3;
  *th = thf;
  *xf = x;
  *yf = y;
  *zf = z;
}

/* ------------------------------------------------------------------------ */
/* Forces at one point for an ion, KineticUpdateA/B/C
 * (_8_1_1_KineticUpdateA.f90:279-944, _8_1_2_KineticUpdateB.f90:128-786,
 * _8_1_3_KineticUpdateC.f90).  Returns the Cartesian acceleration and the
 * geometry used. */
typedef struct {
  double r, th, ph, q, ell, B, Ax, Ay, Az;
} fpoint;

static fpoint force_ion(const orc *o, double x, double y, double z,
                        double Vperp, double AEA, double AG) {
  const kaos_params_c *P = &o->P;
  fpoint f;
  double r = sqrt(x * x + y * y + z * z);
  double th = acos(z / r);
  double ph = o->phiG;
  double ct = cos(th), st = sin(th), cp = cos(ph), sp = sin(ph);
  double q = (RE * RE) * ct / (r * r);
  double ell = 1.0 + 3.0 * (ct * ct);
  double sl = sqrt(ell);
  double B = MDIP * sl / (r * r * r);
  double r4 = r * r * r * r;
  double dBds = (-6.0 * MDIP * ct / r4) - (3.0 * MDIP * ct * (st * st) / (ell * r4));
  double mu = P->ms * (Vperp * Vperp) / (2.0 * B);
  double AMx = 0, AMy = 0, AMz = 0, AGx = 0, AGy = 0, AGz = 0, AEx = 0,
         AEy = 0, AEz = 0;
  if (P->MIRRORflag == 1) { /* :335-365 */
    double AMxp = ((-mu * dBds) * 3.0 * cp * ct * st / sl) / P->ms;
    double AMyp = ((-mu * dBds) * 3.0 * sp * ct * st / sl) / P->ms;
    double AMzp = ((-mu * dBds) * (3.0 * (ct * ct) - 1.0) / sl) / P->ms;
    double proj = 3.0 * ct * st * (AMxp * cp + AMyp * sp) / sl +
                  AMzp * (3.0 * (ct * ct) - 1.0) / sl;
    double AMpar = (q <= 0.0) ? -fabs(proj) : fabs(proj);
    AMx = cp * (3.0 * AMpar * ct * st) / sl;
    AMy = sp * (3.0 * AMpar * ct * st) / sl;
    AMz = AMpar * (3.0 * (ct * ct) - 1.0) / sl;
  }
  if (P->GRAVflag == 1) { /* :478-504 */
    double S = (q <= 0.0) ? 1.0 : -1.0;
    double AGxp = S * fabs(AG) * (3.0 * cp * ct * st / sl);
    double AGyp = S * fabs(AG) * (3.0 * sp * ct * st / sl);
    double AGzp = S * fabs(AG) * ((3.0 * (ct * ct) - 1.0) / sl);
    double AGpar = (3.0 * ct * st * (AGxp * cp + AGyp * sp) / sl +
                    AGzp * (3.0 * (ct * ct) - 1.0) / sl);
    AGx = cp * (3.0 * AGpar * ct * st) / sl;
    AGy = sp * (3.0 * AGpar * ct * st) / sl;
    AGz = AGpar * (3.0 * (ct * ct) - 1.0) / sl;
  }
  if (P->EAMBflag == 1) { /* :646-678, AEA*sub :720-754 */
    double S, mag;
    if (P->EAMBSIGNflag == 0) {
      S = (q <= 0.0) ? -1.0 : 1.0;
      mag = fabs(AEA);
    } else {
      S = 1.0;
      mag = AEA;
    }
    double AExp = S * mag * (3.0 * cp * ct * st / sl);
    double AEyp = S * mag * (3.0 * sp * ct * st / sl);
    double AEzp = S * mag * ((3.0 * (ct * ct) - 1.0) / sl);
    double AEpar = (3.0 * ct * st * (AExp * cp + AEyp * sp) / sl +
                    AEzp * (3.0 * (ct * ct) - 1.0) / sl);
    AEx = cp * (3.0 * AEpar * ct * st) / sl;
    AEy = sp * (3.0 * AEpar * ct * st) / sl;
    AEz = AEpar * (3.0 * (ct * ct) - 1.0) / sl;
  }
  /* parallel potential structure: EPARflag = 0 in every configuration */
  f.Ax = AMx + AGx + AEx + 0.0;
  f.Ay = AMy + AGy + AEy + 0.0;
  f.Az = AMz + AGz + AEz + 0.0;
  f.r = r;
  f.th = th;
  f.ph = ph;
  f.q = q;
  f.ell = ell;
  f.B = B;
  return f;
}

/* ENA forces: gravity only, AGENA*sub _KineticMainParams.f90:695-714. */
static fpoint force_ena(const orc *o, double x, double y, double z) {
  fpoint f;
  double r = sqrt(x * x + y * y + z * z);
  double th = acos(z / r);
  double ph = atan2(y, x);
  f.r = r;
  f.th = th;
  f.ph = ph;
  f.q = (RE * RE) * cos(th) / (r * r);
  f.ell = 1.0 + 3.0 * sq(cos(th));
  f.B = 0.0;
  if (o->P.GRAVflag == 1) {
    double mN = o->P.mNeut;
    f.Ax = ((-GG * ME * mN / (r * r)) * sin(th) * cos(ph)) / mN;
    f.Ay = ((-GG * ME * mN / (r * r)) * sin(th) * sin(ph)) / mN;
    f.Az = ((-GG * ME * mN / (r * r)) * cos(th)) / mN;
  } else {
    f.Ax = f.Ay = f.Az = 0.0;
  }
  return f;
}

/* Gaussian by Box-Muller (GaussianRNGSub _3_1_GaussianRNG.f90:33) from a
 * Philox draw keyed by (id, step, stream, sub). */
static double gauss(uint64_t seed, uint64_t id, uint32_t step, uint32_t stream,
                    uint32_t sub) {
  kaos_u32x4 w = kaos_philox((uint32_t)id, (uint32_t)(id >> 32), step,
                             (stream << 24) | sub, seed);
  double u1 = kaos_u01(w.v[0], w.v[1]);
  double u2 = kaos_u01(w.v[2], w.v[3]);
  return sqrt(-2.0 * log(u1)) * cos(2.0 * PI * u2);
}

/* ------------------------------------------------------------------------ */
/* WaveHeatingSub _8_1_1_0_WaveHeating.f90:24-573 (stochastic branch and
 * coherent branch).  Returns the new Vperp1, Vperp2. */
static void wave_heating(orc *o, int64_t j, int64_t Qk1, double OmegaGk1,
                         double VxR, double VyR, double VzR, double *V1N,
                         double *V2N) {
  const kaos_params_c *P = &o->P;
  *V1N = o->V1[j];
  *V2N = o->V2[j];
  if (!(P->ICRflag == 1 && Qk1 != 0 && Qk1 != -1))
    return;
  int c = (int)Qk1 - 1;
  double lam = o->lambdaPerp[c], eta = o->EtaLH[c], xi1 = o->XiPerp1[c],
         xi2 = o->XiPerp2[c], S0 = o->S0[c], Om0 = o->OmegaG0[c],
         chi1 = o->ChiPerp1[c], chi2 = o->ChiPerp2[c];
  uint32_t step = (uint32_t)o->n;
  /* two Gaussians from one draw: both Box-Muller branches */
  kaos_u32x4 wr = kaos_philox((uint32_t)o->id[j], (uint32_t)(o->id[j] >> 32),
                              step, KAOS_RNG_HEAT << 24, P->seed);
  double R = sqrt(-2.0 * log(kaos_u01(wr.v[0], wr.v[1])));
  double u2 = kaos_u01(wr.v[2], wr.v[3]);
  double G1 = R * cos(2.0 * PI * u2);
  double G2 = R * sin(2.0 * PI * u2);
  double vpm = sqrt(sq(o->V1[j]) + sq(o->V2[j]));
  double Sig = 1.0;
  if ((lam != 0.0) && (((2.0 * PI * vpm) / OmegaGk1) >= lam))
    Sig = (2.0 * PI * vpm) / (lam * OmegaGk1);
  double D1 = ((sq(P->qs) / (2.0 * sq(P->ms))) * (xi1 * eta) * S0 *
               pow(OmegaGk1 / Om0, -chi1)) *
              pow(Sig, -3.0);
  double D2 = ((sq(P->qs) / (2.0 * sq(P->ms))) * (xi2 * eta) * S0 *
               pow(OmegaGk1 / Om0, -chi2)) *
              pow(Sig, -3.0);
  double eps = fabs(sqrt(VxR * VxR + VyR * VyR + VzR * VzR) /
                    (OmegaGk1 * o->sumdsICR));
  double tau = 1.0 / ((OmegaGk1 / (2.0 * PI)) * fabs(sqrt(eps)));
  double h = P->h;
  if (P->ICRCOHERENCEflag == 1) {
    double dV = (h / tau) * sqrt(2.0 * (D1 + D2) * tau) * G1;
    double VpN = o->Vp[j] + dV;
    kaos_u32x4 w = kaos_philox((uint32_t)o->id[j], (uint32_t)(o->id[j] >> 32),
                               step, (KAOS_RNG_HEAT << 24) | 2u, P->seed);
    double ga = kaos_u01(w.v[0], w.v[1]) * 2.0 * PI;
    /* quadrant reconstruction :183-298 == (|V| cos ga, |V| sin ga) */
    *V1N = fabs(VpN) * cos(ga);
    *V2N = fabs(VpN) * sin(ga);
  } else {
    double d1 = 0.0, d2 = 0.0;
    if (h <= tau) {
      d1 = (h / tau) * sqrt(2.0 * D1 * tau) * G1;
      d2 = (h / tau) * sqrt(2.0 * D2 * tau) * G2;
    }
    *V1N = o->V1[j] + d1;
    *V2N = o->V2[j] + d2;
  }
}

/* ENA velocity-bin search, KineticUpdateA _8_1_1_KineticUpdateA.f90:1161-
 * 1230 (1-based): the first cell is [lo,hi], later cells (lo,hi].  The
 * reference's out-of-grid test (lowest edge > v and v > highest edge) can
 * never hold, so a value outside the grid keeps the previous index. */
static int64_t ena_bin(const double *e, int n, double v, int64_t prev) {
  for (int k = 1; k <= n; ++k) {
    if (k == 1 ? (e[0] <= v && v <= e[1]) : (e[k - 1] < v && v <= e[k]))
      return k;
  }
  return prev;
}

/* ------------------------------------------------------------------------ */
/* KineticRK4UpdateSub _8_1_KineticRK4Update.f90:29-315 for particle j;
 * KineticUpdateA's binning indices (:221-273, :988-1129) are stored. */
static void push_particle(orc *o, int64_t j) {
  const kaos_params_c *P = &o->P;
  const double h = P->h;
  int isena = o->ena[j];
  double x = o->x[j], y = o->y[j], z = o->z[j];
  fpoint k1 = isena ? force_ena(o, x, y, z)
                    : force_ion(o, x, y, z, o->Vp[j], o->AEA[j], o->AG[j]);
  double ct = cos(k1.th), st = sin(k1.th), cp = cos(k1.ph), sp = sin(k1.ph);
  double sl = sqrt(k1.ell);
  {
    int64_t Qs = cell_search(o, k1.q);
    if (Qs != -9)
      o->Qind[j] = Qs;
  }
  /* Vpar projection :978-980 */
  double Vpar = 3.0 * ct * st * (o->Vx[j] * cp + o->Vy[j] * sp) / sl +
                o->Vz[j] * (3.0 * (ct * ct) - 1.0) / sl;
  double Vpv = 0.0, Vphv = 0.0;
  if (!isena) {
    if (P->ION2VPERPflag == 1) {
      o->ipar[j] = vbin(o->epar, o->npar, Vpar, 1, o->ipar[j]);
      o->i1[j] = vbin(o->e1, o->n1, o->V1[j], 1, o->i1[j]);
      o->i2[j] = vbin(o->e2, o->n2, o->V2[j], 1, o->i2[j]);
    } else {
      o->ipar[j] = vbin(o->epar, o->npar, Vpar, 0, o->ipar[j]);
      o->i1[j] = vbin(o->e1, o->n1, o->Vp[j], 0, o->i1[j]);
    }
  } else {
    if (o->Qind[j] != -1 && o->Qind[j] != 0) { /* :1155-1160 */
      o->Vpe[j] = fabs((1.0 - 3.0 * (ct * ct)) * (o->Vx[j] * cp + o->Vy[j] * sp) / sl +
                       3.0 * o->Vz[j] * ct * st / sl);
      o->Vphe[j] = -o->Vx[j] * sp + o->Vy[j] * cp;
      o->iep[j] = ena_bin(o->eep, o->nep, o->Vpe[j], o->iep[j]);
      o->ieq[j] = ena_bin(o->eeq, o->neq, Vpar, o->ieq[j]);
      o->ieph[j] = ena_bin(o->eeph, o->neph, o->Vphe[j], o->ieph[j]);
    }
    Vpv = o->Vpe[j];
    Vphv = o->Vphe[j];
  }
  /* field-aligned Cartesian velocity :1327-1334 */
  double VxR = cp * (3.0 * Vpar * ct * st + Vpv * (1.0 - 3.0 * (ct * ct))) / sl -
               Vphv * sp;
  double VyR = sp * (3.0 * Vpar * ct * st + Vpv * (1.0 - 3.0 * (ct * ct))) / sl +
               Vphv * cp;
  double VzR = Vpar * (3.0 * (ct * ct) - 1.0) / sl + 3.0 * Vpv * ct * st / sl;
  /* wave heating :1392 (uses Qindk1 of this step) */
  double V1N = o->V1[j], V2N = o->V2[j];
  if (!isena) {
    double OmegaGk1 = P->qs * k1.B / P->ms;
    wave_heating(o, j, o->Qind[j], OmegaGk1, VxR, VyR, VzR, &V1N, &V2N);
  }
  /* k2 :39-47 */
  double xk2 = x + (h / 2.0) * VxR;
  double yk2 = y + (h / 2.0) * VyR;
  double zk2 = z + (h / 2.0) * VzR;
  fpoint k2 = isena ? force_ena(o, xk2, yk2, zk2)
                    : force_ion(o, xk2, yk2, zk2, o->Vp[j], o->AEA[j], o->AG[j]);
  /* k4 :66-71 */
  double xk4 = x + h * VxR + ((h * h) / 2.0) * k1.Ax;
  double yk4 = y + h * VyR + ((h * h) / 2.0) * k1.Ay;
  double zk4 = z + h * VzR + ((h * h) / 2.0) * k1.Az;
  fpoint k4 = isena ? force_ena(o, xk4, yk4, zk4)
                    : force_ion(o, xk4, yk4, zk4, o->Vp[j], o->AEA[j], o->AG[j]);
  /* KineticUpdateC stores the k4 geometry (_8_1_3_KineticUpdateC.f90:31-62) */
  o->qk4[j] = k4.q;
  o->rk4[j] = k4.r;
  o->thk4[j] = k4.th;
  o->phk4[j] = k4.ph;
  o->ellk4[j] = k4.ell;
  /* velocity RK combination :85-90 (k3 = k2) */
  double VxNp = VxR + (h / 6.0) * (k1.Ax + 2.0 * k2.Ax + 2.0 * k2.Ax + k4.Ax);
  double VyNp = VyR + (h / 6.0) * (k1.Ay + 2.0 * k2.Ay + 2.0 * k2.Ay + k4.Ay);
  double VzNp = VzR + (h / 6.0) * (k1.Az + 2.0 * k2.Az + 2.0 * k2.Az + k4.Az);
  /* position RK combination :124-146 */
  double k1x = VxR, k1y = VyR, k1z = VzR;
  double Vxk2 = VxR + (h / 2.0) * k1.Ax, Vyk2 = VyR + (h / 2.0) * k1.Ay,
         Vzk2 = VzR + (h / 2.0) * k1.Az;
  double Vxk4 = VxR + h * k2.Ax, Vyk4 = VyR + h * k2.Ay, Vzk4 = VzR + h * k2.Az;
  double xN, yN, zN;
  if (!isena) { /* :151-176 */
    double xNp = x + (h / 6.0) * (k1x + 2.0 * Vxk2 + 2.0 * Vxk2 + Vxk4);
    double yNp = y + (h / 6.0) * (k1y + 2.0 * Vyk2 + 2.0 * Vyk2 + Vyk4);
    double zNp = z + (h / 6.0) * (k1z + 2.0 * Vzk2 + 2.0 * Vzk2 + Vzk4);
    double rNp = sqrt(xNp * xNp + yNp * yNp + zNp * zNp);
    double thNp = acos(zNp / rNp);
    double qNp = (RE * RE) * cos(thNp) / (rNp * rNp);
    double rr, tt;
    quartic(qNp, o->pG, o->phiG, &rr, &tt, &xN, &yN, &zN);
  } else { /* :186-193 */
    xN = x + (h / 6.0) * (k1x + 2.0 * Vxk2 + 2.0 * Vxk2 + Vxk4);
    yN = y + (h / 6.0) * (k1y + 2.0 * Vyk2 + 2.0 * Vyk2 + Vyk4);
    zN = z + (h / 6.0) * (k1z + 2.0 * Vzk2 + 2.0 * Vzk2 + Vzk4);
  }
  /* re-align velocity :227-315 */
  double rN = sqrt(xN * xN + yN * yN + zN * zN);
  double thN = acos(zN / rN);
  double phN = isena ? atan2(yN, xN) : o->phiG;
  double ctN = cos(thN), stN = sin(thN), cpN = cos(phN), spN = sin(phN);
  double ellN = 1.0 + 3.0 * (ctN * ctN);
  double slN = sqrt(ellN);
  double VparNp = 3.0 * ctN * stN * (VxNp * cpN + VyNp * spN) / slN +
                  VzNp * (3.0 * (ctN * ctN) - 1.0) / slN;
  double VpNp = 0.0, VphiNp = 0.0;
  if (isena) {
    VpNp = fabs((1.0 - 3.0 * (ctN * ctN)) * (VxNp * cpN + VyNp * spN) / slN +
                3.0 * VzNp * ctN * stN / slN);
    VphiNp = -VxNp * spN + VyNp * cpN;
  }
  o->Vx[j] = cpN * (3.0 * VparNp * ctN * stN + VpNp * (1.0 - 3.0 * (ctN * ctN))) / slN -
             VphiNp * spN;
  o->Vy[j] = spN * (3.0 * VparNp * ctN * stN + VpNp * (1.0 - 3.0 * (ctN * ctN))) / slN +
             VphiNp * cpN;
  o->Vz[j] = VparNp * (3.0 * (ctN * ctN) - 1.0) / slN + 3.0 * VpNp * ctN * stN / slN;
  o->x[j] = xN;
  o->y[j] = yN;
  o->z[j] = zN;
  if (!isena) {
    o->V1[j] = V1N;
    o->V2[j] = V2N;
    o->Vp[j] = fabs(sqrt(V1N * V1N + V2N * V2N));
  }
}

/* ------------------------------------------------------------------------ */
/* MomentFilterSub _8_7_1_MomentFilter.f90:25-147 (0-based cells 0..nq-1) */
static void moment_filter(const double *in, double *out, int nq, int Pt) {
  int H = (int)lround((Pt - 1.0) / 2.0);
  int LB = 0, UB = nq - 1;
  for (int Q = 0; Q < nq; ++Q) {
    double s1, s2, a1, a2;
    if (Q <= LB - 1 + H) {
      s1 = in[Q] + in[Q + 1];
      for (int k = 2; k <= H; ++k)
        s1 += in[Q + k];
      a1 = s1 / (H + 1);
      if (Q == LB)
        out[Q] = a1;
      else if (Q == LB + 1)
        out[Q] = (a1 + in[LB]) / 2.0;
      else {
        s2 = in[Q - 1];
        for (int k = 2; k <= Q - LB; ++k)
          s2 += in[Q - k];
        a2 = s2 / (Q - LB);
        out[Q] = (a1 + a2) / 2.0;
      }
    }
    if ((Q > LB - 1 + H) && (Q < UB - H)) {
      s1 = in[Q] + in[Q + 1];
      for (int k = 2; k <= H; ++k)
        s1 += in[Q + k];
      s2 = in[Q - 1];
      for (int k = 2; k <= H; ++k)
        s2 += in[Q - k];
      a1 = s1 / (H + 1);
      a2 = s2 / H;
      out[Q] = (a1 + a2) / 2.0;
    }
    if (Q >= UB - H) {
      s2 = in[Q] + in[Q - 1];
      for (int k = 2; k <= H; ++k)
        s2 += in[Q - k];
      a2 = s2 / (H + 1);
      if (Q == UB)
        out[Q] = a2;
      else if (Q == UB - 1)
        out[Q] = (in[UB] + a2) / 2.0;
      else {
        s1 = in[Q + 1];
        for (int k = 2; k <= UB - Q; ++k)
          s1 += in[Q + k];
        a1 = s1 / (UB - Q);
        out[Q] = (a1 + a2) / 2.0;
      }
    }
  }
}

/* AmbipolarEfieldSub pressure term _8_7_AmbipolarEfield.f90:611-1299 with
 * MOMENTFILTERflag as given; M0prev = M0phRT(nn-1,:), M0f = filtered. */
static void ambipolar(orc *o, const double *M0prev) {
  const kaos_params_c *P = &o->P;
  int nq = o->nq;
  double *M0f = o->mom[KAOS_M0FILT];
  if (P->MOMENTFILTERflag == 1)
    moment_filter(M0prev, M0f, nq, P->M0MAfilterPt);
  else
    memcpy(M0f, M0prev, sizeof(double) * (size_t)nq);
  const double *Mn = M0f;
  double S = (o->qGL[0] <= 0.0) ? 1.0 : -1.0; /* sign of the denominators */
  double *EP = (double *)calloc((size_t)nq, sizeof(double));
  for (int Q = 0; Q < nq; ++Q) {
    if (!(M0prev[Q] != 0.0 && P->EAPRESSUREflag == 1))
      continue;
    double R1 = (1.0 / fabs(o->hqC[Q])) * (KB * o->Te[Q] / (P->qs * Mn[Q]));
    double st, den;
    if (Q == 0) {
      st = -25.0 * Mn[Q] + 48.0 * Mn[Q + 1] - 36.0 * Mn[Q + 2] +
           16.0 * Mn[Q + 3] - 3.0 * Mn[Q + 4];
      den = 12.0 * o->dqC[Q];
    } else if (Q == nq - 1) {
      st = -25.0 * Mn[Q] + 48.0 * Mn[Q - 1] - 36.0 * Mn[Q - 2] +
           16.0 * Mn[Q - 3] - 3.0 * Mn[Q - 4];
      den = -12.0 * o->dqC[Q];
    } else if (Q == 1 || Q == nq - 2) {
      st = Mn[Q + 1] - Mn[Q - 1];
      den = 2.0 * o->dqC[Q];
    } else {
      st = Mn[Q - 2] - 8.0 * Mn[Q - 1] + 8.0 * Mn[Q + 1] - Mn[Q + 2];
      den = 12.0 * o->dqC[Q];
    }
    double R2;
    if (P->EAMBSIGNflag == 0)
      R2 = fabs(st) / den;
    else
      R2 = -(st) / (-S * den);
    double R = R1 * R2;
    EP[Q] = (P->EAMBSIGNflag == 0) ? fabs(R) : R;
  }
  if (P->EAMBSELFCONSISTflag == 1) /* LB cutoff :1276-1284 */
    for (int Q = 0; Q <= 2 && Q < nq; ++Q)
      if (M0prev[Q] != 0.0 && P->EAPRESSUREflag == 1 && nq > 3)
        EP[Q] = EP[3];
  for (int Q = 0; Q < nq; ++Q)
    o->EAmag[Q] = 0.0 + EP[Q]; /* EAInertial = 0 (EAINERTIALflag = 0) */
  free(EP);
}

/* GravfieldSub E_G at cell centres _8_7_2_Gravfield.f90:57-65 */
static void gravfield(orc *o) {
  const kaos_params_c *P = &o->P;
  for (int Q = 0; Q < o->nq; ++Q)
    o->EG[Q] = (P->GRAVflag == 1)
                   ? (-2.0 * GG * ME * P->ms * cos(o->thetaGC[Q]) /
                      (P->qs * (o->rGC[Q] * o->rGC[Q]) * sqrt(o->ellGC[Q])))
                   : 0.0;
}

/* Per-particle field interpolation between cell centres at q
 * (_8_7_AmbipolarEfield.f90:1453-2722, _8_7_2_Gravfield.f90:132-...).
 * Returns 0 if q lies outside the grid (value unchanged). */
static int interp_field(const orc *o, const double *E, double q, double *out) {
  ORC_SEARCH_BEGIN(); /* the orientation products stand for branches */
  double s = orient(o);
  double sq_ = s * q;
  int nq = o->nq;
  int found = 0, lerp = 0, at = 0;
  for (int Q = 0; Q < nq && !found; ++Q) {
    double cQ = s * o->qGC[Q];
    if (Q == 0 && s * o->qGL[0] <= sq_ && sq_ <= cQ) {
      found = 1;
      at = 0;
    } else if (Q != 0 && Q != nq - 1 && s * o->qGC[Q - 1] < sq_ && sq_ <= cQ) {
      found = lerp = 1;
      at = Q;
    } else if (Q == nq - 1) {
      if (s * o->qGC[Q - 1] < sq_ && sq_ < cQ) {
        found = lerp = 1;
        at = Q;
      } else if (cQ <= sq_ && sq_ <= s * o->qGH[Q]) {
        found = 1;
        at = Q;
      }
    }
  }
  ORC_SEARCH_END();
  if (found)
    *out = lerp ? lin_interp(q, E[at - 1], E[at], o->qGC[at - 1], o->qGC[at])
                : E[at];
  return found;
}

static void interpolate_particles(orc *o, int use_q0, const double *q0) {
  const kaos_params_c *P = &o->P;
  double qm = P->qs / P->ms;
  for (int64_t j = 0; j < o->np; ++j) {
    if (o->ena[j])
      continue;
    double q = use_q0 ? q0[j] : o->qk4[j];
    double v;
    if (P->EAMBflag == 1 && interp_field(o, o->EAmag, q, &v)) {
      double e = (P->EAMBSIGNflag == 0) ? fabs(v) : v;
      o->AEAN[j] = (e == 0.0) ? 0.0
                              : ((P->EAMBSIGNflag == 0) ? fabs(qm * e) : qm * e);
    }
    if (P->GRAVflag == 1 && interp_field(o, o->EG, q, &v)) {
      double e = fabs(v);
      o->AGN[j] = (e == 0.0) ? 0.0 : fabs(qm * e);
    }
  }
}

/* The one occupied bin of axis `ax` (0: Vperp1, 1: Vperp2, 2: Vpar) of a
 * cell's histogram H[(i1*n2 + i2)*npar + ip], or -1 when several are. */
static int single_bin(const int64_t *H, int n1, int n2, int npar, int ax) {
  int found = -1;
  for (int i1 = 0; i1 < n1; ++i1)
    for (int i2 = 0; i2 < n2; ++i2)
      for (int ip = 0; ip < npar; ++ip) {
        if (!H[((int64_t)i1 * n2 + i2) * npar + ip])
          continue;
        int k = ax == 0 ? i1 : (ax == 1 ? i2 : ip);
        if (found >= 0 && found != k)
          return -1;
        found = k;
      }
  return found;
}

/* ------------------------------------------------------------------------ */
/* ParticleCounts / DistributionFunctions / moments for one master step
 * (_8_3_1_IonParticleCounts.f90:26-451, _8_4_1_IonDistributionFunctions
 * .f90:25-163, _8_6_1 ... _8_6_6, NonUniform2D/3D integrators). */
static void statistics(orc *o) {
  const kaos_params_c *P = &o->P;
  int nq = o->nq, nv = o->nv;
  int d3 = (P->ION2VPERPflag == 1);
  memset(o->cnt, 0, sizeof(int64_t) * (size_t)nq);
  memset(o->hist, 0, sizeof(int64_t) * (size_t)nq * (size_t)nv);
  if (o->literal) {
    /* literal O(Nq * Nv * Np) loops :45-80, :311-357, :589-632 */
    for (int Q = 1; Q <= nq; ++Q) {
      int64_t c = 0;
      for (int64_t j = 0; j < o->np; ++j)
        if (!o->ena[j] && o->Qind[j] == Q)
          c++;
      o->cnt[Q - 1] = c;
      if (c == 0)
        continue;
      for (int b = 0; b < nv; ++b) {
        int64_t i1 = d3 ? (b / (o->n2 * o->npar)) + 1 : (b / o->npar) + 1;
        int64_t i2 = d3 ? ((b / o->npar) % o->n2) + 1 : 0;
        int64_t ip = (b % o->npar) + 1;
        int64_t cc = 0;
        for (int64_t j = 0; j < o->np; ++j)
          if (!o->ena[j] && o->i1[j] == i1 && (!d3 || o->i2[j] == i2) &&
              o->ipar[j] == ip && o->Qind[j] == Q)
            cc++;
        o->hist[(int64_t)(Q - 1) * nv + b] = cc;
      }
    }
  } else {
    for (int64_t j = 0; j < o->np; ++j) {
      if (o->ena[j])
        continue;
      int64_t Q = o->Qind[j];
      if (Q < 1 || Q > nq)
        continue;
      o->cnt[Q - 1]++;
      if (o->i1[j] < 1 || o->ipar[j] < 1 || (d3 && o->i2[j] < 1))
        continue;
      int64_t b = d3 ? ((o->i1[j] - 1) * o->n2 + (o->i2[j] - 1)) * o->npar +
                           (o->ipar[j] - 1)
                     : (o->i1[j] - 1) * o->npar + (o->ipar[j] - 1);
      o->hist[(Q - 1) * nv + b]++;
    }
  }
  double ms = P->ms;
  for (int Q = 0; Q < nq; ++Q) {
    double w = o->nsnormfac / o->d3xC[Q];
    double NqRT = (double)o->cnt[Q] * w;
    o->mom[KAOS_NQ][Q] = NqRT;
    for (int k = 0; k <= KAOS_M2PERP; ++k)
      o->mom[k][Q] = 0.0;
    if (NqRT == 0.0)
      continue;
    const int64_t *H = o->hist + (int64_t)Q * nv;
    /* F = N2PerpphRT/d3v with N2PerpphRT = count*nsnormfac/d3x */
#define FBIN(b) ((H[b] == 0) ? 0.0 : ((double)H[b] * w) / o->d3v[b])
    if (d3) {
      /* Fortran sum order: Vperp1 fastest, then Vperp2, then Vpar */
      double S0 = 0, S1 = 0, S2 = 0, Sp = 0;
      for (int ip = 0; ip < o->npar; ++ip)
        for (int i2 = 0; i2 < o->n2; ++i2)
          for (int i1 = 0; i1 < o->n1; ++i1) {
            int b = (i1 * o->n2 + i2) * o->npar + ip;
            double F = FBIN(b);
            double dV = fabs(o->e1[i1 + 1] - o->e1[i1]) * fabs(o->e2[i2 + 1] - o->e2[i2]) *
                 fabs(o->epar[ip + 1] - o->epar[ip]);
            S0 += dV * F;
            S1 += dV * (F == 0.0 ? 0.0 : o->c1[i1] * F);
            S2 += dV * (F == 0.0 ? 0.0 : o->c2[i2] * F);
            Sp += dV * (F == 0.0 ? 0.0 : o->cpar[ip] * F);
          }
      double M0 = S0;
      o->mom[KAOS_M0][Q] = M0;
      if (M0 == 0.0)
        continue;
      double M1p1 = S1 / M0, M1p2 = S2 / M0, M1par = Sp / M0;
      /* a cell whose ions share one bin of an axis has that bin's centre as
       * its first moment along the axis (the exact value of the ratio); the
       * centred second-moment integrand of that bin is then zero and falls
       * back to the uncentred one (_8_6_6_SecondParIonMoment.f90:90-99) */
      int kp = single_bin(H, o->n1, o->n2, o->npar, 2);
      int k1 = single_bin(H, o->n1, o->n2, o->npar, 0);
      int k2 = single_bin(H, o->n1, o->n2, o->npar, 1);
      if (kp >= 0) M1par = o->cpar[kp];
      if (k1 >= 0) M1p1 = o->c1[k1];
      if (k2 >= 0) M1p2 = o->c2[k2];
      o->mom[KAOS_M1PERP1][Q] = M1p1;
      o->mom[KAOS_M1PERP2][Q] = M1p2;
      o->mom[KAOS_M1PAR][Q] = M1par;
      double T = 0, T1 = 0, T2 = 0, Tp = 0;
      for (int ip = 0; ip < o->npar; ++ip)
        for (int i2 = 0; i2 < o->n2; ++i2)
          for (int i1 = 0; i1 < o->n1; ++i1) {
            int b = (i1 * o->n2 + i2) * o->npar + ip;
            double F = FBIN(b);
            double dV = fabs(o->e1[i1 + 1] - o->e1[i1]) * fabs(o->e2[i2 + 1] - o->e2[i2]) *
                        fabs(o->epar[ip + 1] - o->epar[ip]);
            double g = 0, g1 = 0, g2 = 0, gp = 0;
            if (F != 0.0) {
              double vc = o->cpar[ip];
              if (P->PHASEENERGYPARIONMOMENTCENTERflag == 1) {
                g = (sq(o->c1[i1]) + sq(o->c2[i2]) + sq(vc - M1par)) * F;
                if (isnan(g) || g == 0.0)
                  g = (sq(o->c1[i1]) + sq(o->c2[i2]) + sq(vc)) * F;
                gp = sq(vc - M1par) * F;
                if (isnan(gp) || gp == 0.0)
                  gp = sq(vc) * F;
              } else {
                g = (sq(o->c1[i1]) + sq(o->c2[i2]) + sq(vc)) * F;
                gp = sq(vc) * F;
              }
              if (P->PHASEENERGYPERPIONMOMENTCENTERflag == 1) {
                g1 = sq(o->c1[i1] - M1p1) * F;
                if (isnan(g1) || g1 == 0.0)
                  g1 = sq(o->c1[i1]) * F;
                g2 = sq(o->c2[i2] - M1p2) * F;
                if (isnan(g2) || g2 == 0.0)
                  g2 = sq(o->c2[i2]) * F;
              } else {
                g1 = sq(o->c1[i1]) * F;
                g2 = sq(o->c2[i2]) * F;
              }
            }
            T += dV * g;
            T1 += dV * g1;
            T2 += dV * g2;
            Tp += dV * gp;
          }
      o->mom[KAOS_M2][Q] = (ms / 2.0) * (T / M0);
      o->mom[KAOS_M2PERP1][Q] = (ms / 2.0) * (T1 / M0);
      o->mom[KAOS_M2PERP2][Q] = (ms / 2.0) * (T2 / M0);
      o->mom[KAOS_M2PAR][Q] = ((ms / 2.0) * (Tp / M0));
    } else {
      /* 2D cylindrical grid: MM = 2*pi*sum(dVperp*dVpar*g) */
      double S0 = 0, Sperp = 0, Spar = 0;
      for (int ip = 0; ip < o->npar; ++ip)
        for (int i1 = 0; i1 < o->n1; ++i1) {
          int b = i1 * o->npar + ip;
          double F = FBIN(b);
          double dV = fabs(o->e1[i1 + 1] - o->e1[i1]) * fabs(o->epar[ip + 1] - o->epar[ip]);
          double vc = o->c1[i1];
          S0 += dV * (F == 0.0 ? 0.0 : vc * F);
          Sperp += dV * (F == 0.0 ? 0.0 : (vc * vc) * F);
          Spar += dV * (F == 0.0 ? 0.0 : vc * o->cpar[ip] * F);
        }
      double M0 = 2.0 * PI * S0;
      o->mom[KAOS_M0][Q] = M0;
      if (M0 == 0.0)
        continue;
      double M1perp = (2.0 * PI * Sperp) / M0, M1par = (2.0 * PI * Spar) / M0;
      int kp = single_bin(H, o->n1, 1, o->npar, 2);
      int k1 = single_bin(H, o->n1, 1, o->npar, 0);
      if (kp >= 0) M1par = o->cpar[kp];
      if (k1 >= 0) M1perp = o->c1[k1];
      o->mom[KAOS_M1PERP][Q] = M1perp;
      o->mom[KAOS_M1PAR][Q] = M1par;
      double T = 0, Tperp = 0, Tp = 0;
      for (int ip = 0; ip < o->npar; ++ip)
        for (int i1 = 0; i1 < o->n1; ++i1) {
          int b = i1 * o->npar + ip;
          double F = FBIN(b);
          double dV = fabs(o->e1[i1 + 1] - o->e1[i1]) * fabs(o->epar[ip + 1] - o->epar[ip]);
          double vc = o->c1[i1], pc = o->cpar[ip];
          double g = 0, gperp = 0, gp = 0;
          if (F != 0.0) {
            if (P->PHASEENERGYPARIONMOMENTCENTERflag == 1) {
              g = (vc * (vc * vc) * F) + (vc * sq(pc - M1par) * F);
              if (isnan(g) || g == 0.0)
                g = (vc * (vc * vc) * F) + (vc * (pc * pc) * F);
              gp = (vc * sq(pc - M1par) * F);
              if (isnan(gp) || gp == 0.0)
                gp = (vc * (pc * pc) * F);
            } else {
              g = (vc * (vc * vc) * F) + (vc * (pc * pc) * F);
              gp = (vc * (pc * pc) * F);
            }
            if (P->PHASEENERGYPERPIONMOMENTCENTERflag == 1) {
              gperp = (vc * sq(vc - M1perp) * F);
              if (isnan(gperp) || gperp == 0.0)
                gperp = (vc * (vc * vc) * F);
            } else
              gperp = (vc * (vc * vc) * F);
          }
          T += dV * g;
          Tperp += dV * gperp;
          Tp += dV * gp;
        }
      o->mom[KAOS_M2][Q] = (ms / 2.0) * ((2.0 * PI * T) / M0);
      o->mom[KAOS_M2PERP][Q] = (ms / 2.0) * ((2.0 * PI * Tperp) / M0);
      o->mom[KAOS_M2PAR][Q] = ((ms / 2.0) * ((2.0 * PI * Tp) / M0));
    }
#undef FBIN
  }
}

/* IonNeutralCollisionFrequencyASub _8_6_6_1_...:28-301 with the model-A
 * Poisson count clipped to the cell ion count (see DESIGN notes on the
 * rank-split routine B). */
static void collision_frequency(orc *o, uint32_t nn) {
  const kaos_params_c *P = &o->P;
  int nq = o->nq;
  double *m1p = (double *)malloc(sizeof(double) * (size_t)nq);
  double *m11 = (double *)malloc(sizeof(double) * (size_t)nq);
  double *m12 = (double *)malloc(sizeof(double) * (size_t)nq);
  double *m2p = (double *)malloc(sizeof(double) * (size_t)nq);
  int d3 = P->ION2VPERPflag == 1;
  const double *M1P1 = d3 ? o->mom[KAOS_M1PERP1] : o->mom[KAOS_M1PERP];
  const double *M1P2 = o->mom[KAOS_M1PERP2];
  if (P->MOMENTFILTERflag == 1) {
    moment_filter(o->mom[KAOS_M1PAR], m1p, nq, P->M1ParMAfilterPt);
    moment_filter(M1P1, m11, nq, P->M1Perp1MAfilterPt);
    moment_filter(M1P2, m12, nq, P->M1Perp2MAfilterPt);
    moment_filter(o->mom[KAOS_M2PAR], m2p, nq, P->M2ParMAfilterPt);
  } else {
    memcpy(m1p, o->mom[KAOS_M1PAR], sizeof(double) * (size_t)nq);
    memcpy(m11, M1P1, sizeof(double) * (size_t)nq);
    memcpy(m12, M1P2, sizeof(double) * (size_t)nq);
    memcpy(m2p, o->mom[KAOS_M2PAR], sizeof(double) * (size_t)nq);
  }
  for (int Q = 0; Q < nq; ++Q) {
    double sigma = 0.0;
    if (o->mom[KAOS_M0][Q] != 0.0 && m2p[Q] != 0.0)
      sigma = sq(4.07 - 0.269 * log((6.242e18) * (1e-3) * m2p[Q])) *
              pow(1.0 - exp(-415.0 / ((6.242e18) * (1e-3) * m2p[Q])), 0.8);
    double nu = 0.0;
    if (o->mom[KAOS_M0][Q] != 0.0) {
      uint64_t key = ((uint64_t)nn << 32) | (uint32_t)Q;
      double G[3];
      for (int k = 0; k < 3; ++k)
        G[k] = gauss(P->seed, key, 0u, KAOS_RNG_NEUT, (uint32_t)k);
      double sN = sqrt(KB * P->TNeut / P->mNeut);
      double VxN = sN * G[0], VyN = sN * G[1], VzN = sN * G[2];
      double th = o->thetaGC[Q], ph = o->phiG, el = o->ellGC[Q];
      double ct = cos(th), st = sin(th);
      double MVx = cos(ph) * (3.0 * m1p[Q] * ct * st + m11[Q] * (1.0 - 3.0 * (ct * ct))) / sqrt(el) -
                   m12[Q] * sin(ph);
      double MVy = sin(ph) * (3.0 * m1p[Q] * ct * st + m11[Q] * (1.0 - 3.0 * (ct * ct))) / sqrt(el) +
                   m12[Q] * cos(ph);
      double MVz = m1p[Q] * (3.0 * (ct * ct) - 1.0) / sqrt(el) +
                   3.0 * m11[Q] * ct * st / sqrt(el);
      double vrel = fabs(sqrt(sq(fabs(MVx - VxN)) + sq(fabs(MVy - VyN)) + sq(fabs(MVz - VzN))));
      if (sigma != 0.0) {
        double mean = o->nsnormCNeut[Q] * sigma * vrel * P->h;
        /* PoissonRNGSub _3_2_PoissonRNG.f90:31-38 (product of uniforms) */
        double e = exp(-mean), prod = 1.0;
        int64_t k = -1;
        uint32_t it = 0;
        while (prod > e && it < 100000u) {
          kaos_u32x4 w = kaos_philox((uint32_t)Q, nn, it >> 1,
                                     (KAOS_RNG_POIS << 24), P->seed);
          prod *= (it & 1u) ? kaos_u01(w.v[2], w.v[3]) : kaos_u01(w.v[0], w.v[1]);
          k++;
          it++;
        }
        nu = (double)k;
        if (nu > (double)o->cnt[Q])
          nu = (double)o->cnt[Q];
      }
    }
    o->mom[KAOS_NUPOI][Q] = nu;
    o->nuPoi[Q] = nu;
  }
  free(m1p);
  free(m11);
  free(m12);
  free(m2p);
}

/* ------------------------------------------------------------------------ */
static void ensure_cap(orc *o, int64_t need) {
  if (need <= o->cap)
    return;
  int64_t nc = need * 2;
#define GROW(a, T)                                                             \
  o->a = (T *)realloc(o->a, sizeof(T) * (size_t)nc);                          \
  memset(o->a + o->cap, 0, sizeof(T) * (size_t)(nc - o->cap));
  GROW(x, double) GROW(y, double) GROW(z, double) GROW(Vx, double)
  GROW(Vy, double) GROW(Vz, double) GROW(V1, double) GROW(V2, double)
  GROW(Vp, double) GROW(AEA, double) GROW(AG, double) GROW(AEAN, double)
  GROW(AGN, double) GROW(qk4, double) GROW(rk4, double) GROW(thk4, double)
  GROW(phk4, double) GROW(ellk4, double) GROW(Vpe, double) GROW(Vphe, double)
  GROW(Qind, int64_t) GROW(ipar, int64_t) GROW(i1, int64_t) GROW(i2, int64_t)
  GROW(iep, int64_t) GROW(ieq, int64_t) GROW(ieph, int64_t)
  GROW(ena, unsigned char) GROW(id, uint64_t)
#undef GROW
  o->cap = nc;
}

static void copy_particle(orc *o, int64_t d, int64_t s) {
#define C(a) o->a[d] = o->a[s];
  C(x) C(y) C(z) C(Vx) C(Vy) C(Vz) C(V1) C(V2) C(Vp) C(AEA) C(AG) C(AEAN)
  C(AGN) C(qk4) C(rk4) C(thk4) C(phk4) C(ellk4) C(Vpe) C(Vphe) C(Qind)
  C(ipar) C(i1) C(i2) C(iep) C(ieq) C(ieph) C(ena) C(id)
#undef C
}

/* Set one new ion at field-line coordinate q with field-aligned velocity,
 * as the injection (_8_0_0_2_KineticSolverB.f90:203-475) and the initial
 * conditions do: quartic -> Cartesian, V rebuilt from Vpar only. */
static void place_ion(orc *o, int64_t j, double q, double vpar, double v1,
                      double v2) {
  double r, th, x, y, z;
  quartic(q, o->pG, o->phiG, &r, &th, &x, &y, &z);
  double ct = cos(th), st = sin(th), cp = cos(o->phiG), sp = sin(o->phiG);
  double ell = 1.0 + 3.0 * (ct * ct);
  o->x[j] = x;
  o->y[j] = y;
  o->z[j] = z;
  o->Vx[j] = cp * (3.0 * vpar * ct * st) / sqrt(ell);
  o->Vy[j] = sp * (3.0 * vpar * ct * st) / sqrt(ell);
  o->Vz[j] = vpar * (3.0 * (ct * ct) - 1.0) / sqrt(ell);
  o->V1[j] = v1;
  o->V2[j] = v2;
  o->Vp[j] = fabs(sqrt(v1 * v1 + v2 * v2));
  o->ena[j] = 0;
  /* the k4 point of an ion not yet pushed is where it stands: charge
   * exchange may convert an injected ion before its first push (the
   * reference leaves the k4 arrays of reallocated slots unset) */
  o->qk4[j] = q;
  o->rk4[j] = r;
  o->thk4[j] = th;
  o->phk4[j] = o->phiG;
  o->ellk4[j] = ell;
  o->Qind[j] = cell_search(o, q);
  int d3 = o->P.ION2VPERPflag == 1;
  o->ipar[j] = vbin(o->epar, o->npar, vpar, d3, 0);
  o->i1[j] = vbin(o->e1, o->n1, d3 ? v1 : o->Vp[j], d3, 0);
  o->i2[j] = d3 ? vbin(o->e2, o->n2, v2, 1, 0) : 0;
}

/* LB / UB injection on a master step (_8_0_7_BoundaryConditions.f90:743-809,
 * _8_0_0_2_KineticSolverB.f90:195-793, MBVelocityDistributionSub
 * _6_1_MBVelocityDistribution.f90:29-120). */
static void inject(orc *o, int ub) {
  const kaos_params_c *P = &o->P;
  int Q = ub ? o->nq - 1 : 0;
  int64_t k = (int64_t)llround(ub ? o->nsnormCUB : o->nsnormCLB);
  if (k <= 0)
    return;
  ensure_cap(o, o->np + k);
  double qm = P->qs / P->ms;
  double r, th, x, y, z;
  quartic(o->qGC[Q], o->pG, o->phiG, &r, &th, &x, &y, &z);
  double ct = cos(th), st = sin(th), cp = cos(o->phiG), sp = sin(o->phiG);
  double ell = 1.0 + 3.0 * (ct * ct);
  double sig = sqrt(KB * o->TsG[Q] / P->ms);
  for (int64_t i = 0; i < k; ++i) {
    int64_t j = o->np++;
    uint64_t id = o->next_id++;
    o->id[j] = id;
    double G0 = gauss(P->seed, id, 0u, KAOS_RNG_INJECT, 0);
    double G1 = gauss(P->seed, id, 0u, KAOS_RNG_INJECT, 1);
    double G2 = gauss(P->seed, id, 0u, KAOS_RNG_INJECT, 2);
    double Vx0 = sig * G0, Vy0 = sig * G1, Vz0 = sig * G2;
    double Vp0 = ((1.0 - 3.0 * (ct * ct)) / sqrt(ell)) * (Vx0 * cp + Vy0 * sp) +
                 ((3.0 * Vz0 * ct * st) / sqrt(ell));
    double Vq0 = ((3.0 * ct * st) / sqrt(ell)) * (Vx0 * cp + Vy0 * sp) +
                 ((Vz0 * (3.0 * (ct * ct) - 1.0)) / sqrt(ell));
    double Vph0 = -Vx0 * sp + Vy0 * cp;
    double v1 = Vp0, v2 = Vph0, vpar = Vq0;
    if (P->FLUXINJECTIONflag == 1) { /* Maxwellian flux into the tube */
      kaos_u32x4 w = kaos_philox((uint32_t)id, (uint32_t)(id >> 32), 0u,
                                 (KAOS_RNG_INJECT << 24) | 3u, P->seed);
      double r = sig * sqrt(-2.0 * log(kaos_u01(w.v[0], w.v[1])));
      vpar = ub ? -r : r;
    }
    if (P->STATICINJECTIONflag == 1)
      v1 = v2 = vpar = 0.0;
    place_ion(o, j, o->qGC[Q], vpar, v1, v2);
    o->AEA[j] = fabs(qm * fabs(o->EAmag[Q]));
    o->AG[j] = fabs(qm * fabs(o->EG[Q]));
    o->AEAN[j] = o->AEA[j];
    o->AGN[j] = o->AG[j];
  }
  if (ub)
    o->ub_in = k;
  else
    o->lb_in = k;
}

/* BoundaryConditionsSub escape masks + BCReIndexSub order-preserving pack
 * (_8_0_7_BoundaryConditions.f90:158-503, _8_0_7_1_BCReIndex.f90:33-241). */
static void boundary(orc *o) {
  int64_t w = 0, lb = 0, ub = 0, lbe = 0, ube = 0;
  for (int64_t j = 0; j < o->np; ++j) {
    int esc = (o->Qind[j] == 0 || o->Qind[j] == -1);
    if (esc && !o->ena[j]) {
      if (o->Qind[j] == 0)
        lb++;
      else
        ub++;
    }
    if (esc && o->ena[j]) { /* ENA escape counts :305-416 */
      if (o->Qind[j] == 0)
        lbe++;
      else
        ube++;
    }
    if (!esc) {
      if (w != j)
        copy_particle(o, w, j);
      w++;
    }
  }
  o->np = w;
  o->lb_out = lb;
  o->ub_out = ub;
  o->lbe_out = lbe;
  o->ube_out = ube;
}

/* charge exchange on step n (_8_KineticSolver.f90:95-166,
 * IonNeutralCollisionsSub _8_1_1_1_IonNeutralCollisions.f90:25-58) */
static void charge_exchange(orc *o) {
  for (int Q = 1; Q <= o->nq; ++Q) {
    int64_t N = (int64_t)llround(o->nuPoi[Q - 1]);
    if (!(o->nuPoi[Q - 1] > 0.0))
      continue;
    int64_t cnt = 0;
    for (int64_t j = 0; j < o->np && cnt < N; ++j) {
      if (o->ena[j] || o->Qind[j] != Q)
        continue;
      double th = o->thk4[j], ph = o->phk4[j], el = o->ellk4[j];
      double ct = cos(th), st = sin(th), cp = cos(ph), sp = sin(ph);
      double Vpp = o->V1[j], Vphip = o->V2[j];
      double Vparp = 3.0 * ct * st * (o->Vx[j] * cp + o->Vy[j] * sp) / sqrt(el) +
                     o->Vz[j] * (3.0 * (ct * ct) - 1.0) / sqrt(el);
      o->Vx[j] = cp * (3.0 * Vparp * ct * st + Vpp * (1.0 - 3.0 * (ct * ct))) / sqrt(el) -
                 Vphip * sp;
      o->Vy[j] = sp * (3.0 * Vparp * ct * st + Vpp * (1.0 - 3.0 * (ct * ct))) / sqrt(el) +
                 Vphip * cp;
      o->Vz[j] = Vparp * (3.0 * (ct * ct) - 1.0) / sqrt(el) +
                 3.0 * Vpp * ct * st / sqrt(el);
      o->V1[j] = o->V2[j] = o->Vp[j] = 0.0;
      o->ena[j] = 1;
      o->Vpe[j] = 0.0; /* Vp(j), Vphi(j) still hold the ion zeros */
      o->Vphe[j] = 0.0;
      cnt++;
    }
  }
}

/* ENAParticleCountsSub (_8_3_2_ENAParticleCounts.f90:26-300, counts by
 * Qindk1 and Vp/Vq/Vphi indk1, density units nsnormfac/d3x) and the ENA
 * moments ZerothENAMoment .. SecondPHIENAMoment (_8_10_1 .. _8_10_8):
 * integrands hVp hVq hVphi F (.) at the V3CellT bin centres, M1 = MM/M0,
 * M2 = 6.242e18 (ms/2) MM/M0 with the integrand centred on M1.  The bin
 * sums are taken ENA by ENA (the same terms as the reference's bin loop,
 * one per ENA).  Noise filter off (ENANOISEflag = 0). */
static void ena_statistics(orc *o) {
  const double ms = o->P.ms, eV = 6.242e18;
  for (int Q = 1; Q <= o->nq; ++Q) {
    const double w = o->nsnormfac / o->d3xC[Q - 1];
    int64_t cnt = 0, nval = 0;
    double sp = 0.0, sq_ = 0.0, sph = 0.0;
    for (int64_t j = 0; j < o->np; ++j) {
      if (!o->ena[j] || o->Qind[j] != Q)
        continue;
      cnt++;
      if (o->iep[j] < 1 || o->ieq[j] < 1 || o->ieph[j] < 1)
        continue;
      nval++;
      sp += w * (o->eep[o->iep[j] - 1] + o->eep[o->iep[j]]) / 2.0;
      sq_ += w * (o->eeq[o->ieq[j] - 1] + o->eeq[o->ieq[j]]) / 2.0;
      sph += w * (o->eeph[o->ieph[j] - 1] + o->eeph[o->ieph[j]]) / 2.0;
    }
    const double NqENA = (double)cnt * w;
    double M0 = (NqENA == 0.0) ? 0.0 : (double)nval * w;
    double m1p = 0, m1q = 0, m1ph = 0, t = 0, tp = 0, tq = 0, tph = 0;
    if (M0 != 0.0) {
      m1p = sp / M0;
      m1q = sq_ / M0;
      m1ph = sph / M0;
      for (int64_t j = 0; j < o->np; ++j) {
        if (!o->ena[j] || o->Qind[j] != Q || o->iep[j] < 1 || o->ieq[j] < 1 ||
            o->ieph[j] < 1)
          continue;
        const double cp = (o->eep[o->iep[j] - 1] + o->eep[o->iep[j]]) / 2.0;
        const double cq = (o->eeq[o->ieq[j] - 1] + o->eeq[o->ieq[j]]) / 2.0;
        const double cph = (o->eeph[o->ieph[j] - 1] + o->eeph[o->ieph[j]]) / 2.0;
        const double dp = fabs(sq(m1p - cp)), dq = fabs(sq(m1q - cq)),
                     dph = fabs(sq(m1ph - cph));
        t += w * (dp + dq + dph);
        tp += w * dp;
        tq += w * dq;
        tph += w * dph;
      }
    }
    o->mom[KAOS_ENA_NQ][Q - 1] = NqENA;
    o->mom[KAOS_ENA_M0][Q - 1] = M0;
    o->mom[KAOS_ENA_M1P][Q - 1] = m1p;
    o->mom[KAOS_ENA_M1Q][Q - 1] = m1q;
    o->mom[KAOS_ENA_M1PHI][Q - 1] = m1ph;
    o->mom[KAOS_ENA_M2][Q - 1] = M0 != 0.0 ? eV * (ms / 2.0) * (t / M0) : 0.0;
    o->mom[KAOS_ENA_M2P][Q - 1] = M0 != 0.0 ? eV * (ms / 2.0) * (tp / M0) : 0.0;
    o->mom[KAOS_ENA_M2Q][Q - 1] = M0 != 0.0 ? eV * (ms / 2.0) * (tq / M0) : 0.0;
    o->mom[KAOS_ENA_M2PHI][Q - 1] = M0 != 0.0 ? eV * (ms / 2.0) * (tph / M0) : 0.0;
  }
}

/* ConvectionSub _8_11_Convection.f90:135-258 for a move of the tube to
 * o->pending (new pG/phiG, same q grid): every ion keeps q, moves to the new
 * field line (RK4DipolePolynomialSolverSub at (q, pN, phiN)), keeps its
 * magnetic moment (musub, :146-147, :184-185) and gyro-angle (:168-182,
 * :188-214, the angle of the previous ion kept when a component is exactly
 * zero), and its velocity is rebuilt along the new field direction from
 * VparConvSign |V| (:229-255).  ENAs are left in place (the reference's ENA
 * branch uses the theta and ell of the previous ion, :232-238).  Then the
 * tube's tables are replaced, its evolving Te kept. */
static double bmag(double r, double th) {
  return MDIP * sqrt(1.0 + 3.0 * sq(cos(th))) / (r * r * r);
}

static void convection(orc *o) {
  const kaos_tube_c *t = o->pending;
  const double pN = t->pG, phN = t->phiG, ms = o->P.ms;
  for (int64_t j = 0; j < o->np; ++j) {
    if (o->ena[j])
      continue;
    double r1 = sqrt(o->x[j] * o->x[j] + o->y[j] * o->y[j] + o->z[j] * o->z[j]);
    double th1 = acos(o->z[j] / r1);
    double q = (RE * RE) * cos(th1) / (r1 * r1);
    double ph1 = atan2(o->y[j], o->x[j]);
    double el1 = 1.0 + 3.0 * sq(cos(th1));
    double mu = ms * sq(o->Vp[j]) / (2.0 * bmag(r1, th1));
    /* V|| sign along the old field direction */
    double ct1 = cos(th1), st1 = sin(th1), cp1 = cos(ph1), sp1 = sin(ph1);
    double vpar1 = 3.0 * ct1 * st1 * (o->Vx[j] * cp1 + o->Vy[j] * sp1) / sqrt(el1) +
                   o->Vz[j] * (3.0 * (ct1 * ct1) - 1.0) / sqrt(el1);
    double vmag = sqrt(sq(o->Vx[j]) + sq(o->Vy[j]) + sq(o->Vz[j]));
    double vpar2 = (vpar1 < 0.0 ? -1.0 : 1.0) * fabs(vmag);
    double r2, th2, x, y, z;
    quartic(q, pN, phN, &r2, &th2, &x, &y, &z);
    o->x[j] = x;
    o->y[j] = y;
    o->z[j] = z;
    double V1 = o->V1[j], V2 = o->V2[j];
    if (V1 > 0.0 && V2 > 0.0)
      o->GAconv = atan(fabs(V2) / fabs(V1));
    if (V1 < 0.0 && V2 > 0.0)
      o->GAconv = PI - atan(fabs(V2) / fabs(V1));
    if (V1 < 0.0 && V2 < 0.0)
      o->GAconv = PI + atan(fabs(V2) / fabs(V1));
    if (V1 > 0.0 && V2 < 0.0)
      o->GAconv = 2.0 * PI - atan(fabs(V2) / fabs(V1));
    double GA = o->GAconv;
    double Vpn = sqrt(2.0 * bmag(r2, th2) * mu / ms);
    o->Vp[j] = Vpn;
    if (0.0 < GA && GA <= PI / 2.0) {
      o->V1[j] = fabs(Vpn * cos(GA));
      o->V2[j] = fabs(Vpn * sin(GA));
    }
    if (PI / 2.0 < GA && GA <= PI) {
      o->V1[j] = -fabs(Vpn * cos(PI - GA));
      o->V2[j] = fabs(Vpn * sin(PI - GA));
    }
    if (PI < GA && GA <= 3.0 * PI / 2.0) {
      o->V1[j] = -fabs(Vpn * cos(GA - PI));
      o->V2[j] = -fabs(Vpn * sin(GA - PI));
    }
    if (3.0 * PI / 2.0 < GA && GA <= 2.0 * PI) {
      o->V1[j] = fabs(Vpn * cos(2.0 * PI - GA));
      o->V2[j] = -fabs(Vpn * sin(2.0 * PI - GA));
    }
    double ct = cos(th2), st = sin(th2), el = 1.0 + 3.0 * ct * ct;
    o->Vx[j] = cos(phN) * (3.0 * vpar2 * ct * st) / sqrt(el);
    o->Vy[j] = sin(phN) * (3.0 * vpar2 * ct * st) / sqrt(el);
    o->Vz[j] = vpar2 * (3.0 * (ct * ct) - 1.0) / sqrt(el);
  }
  o->pG = t->pG;
  o->phiG = t->phiG;
  o->nsnormfac = t->nsnormfac;
  o->nsnormCLB = t->nsnormCLB;
  o->nsnormCUB = t->nsnormCUB;
  o->sumdsICR = t->sumdsICR;
  int nq = o->nq;
#define R(a)                                                                   \
  if (t->a)                                                                    \
    memcpy(o->a, t->a, sizeof(double) * (size_t)nq);
  R(qGC) R(hqC) R(dqC) R(d3xC) R(rGC) R(thetaGC) R(ellGC) R(TeG) R(TsG)
  R(nsnormCNeut) R(lambdaPerp) R(EtaLH) R(XiPerp1) R(XiPerp2) R(S0) R(OmegaG0)
  R(ChiPerp1) R(ChiPerp2)
#undef R
}

static int is_master(const orc *o, int64_t n) {
  if (n < 2)
    return 0;
  return (n % o->P.ndatfac) == 0;
}

/* one computational step n = o->n + 1 (_8_KineticSolver.f90:54-239) */
static void step_once(orc *o) {
  const kaos_params_c *P = &o->P;
  int64_t n = o->n + 1;
  o->n = n; /* RNG step key = n */
  ORC_PHASE(ORC_PH_MASTER);
  if (n == 1) {
    /* KineticSolverASub _8_0_0_1_KineticSolverA.f90:43-404: counts and
     * moments from the initial indices, fields, then push from x0. */
    for (int Q = 0; Q < o->nq; ++Q)
      o->Te[Q] = o->TeG[Q];
    statistics(o);
    gravfield(o);
    if (o->have_import)
      memcpy(o->EAmag, o->EAimport, sizeof(double) * (size_t)o->nq);
    else if (P->EAMBflag == 1)
      ambipolar(o, o->mom[KAOS_M0]);
    double *q0 = (double *)malloc(sizeof(double) * (size_t)(o->np + 1));
    for (int64_t j = 0; j < o->np; ++j)
      q0[j] = o->qk4[j];
    interpolate_particles(o, 1, q0);
    free(q0);
    if (P->QEXCHANGEflag == 1)
      collision_frequency(o, 1);
    memcpy(o->M0prev, o->mom[KAOS_M0], sizeof(double) * (size_t)o->nq);
    memcpy(o->mom[KAOS_EAMAG], o->EAmag, sizeof(double) * (size_t)o->nq);
    memcpy(o->mom[KAOS_EGMAG], o->EG, sizeof(double) * (size_t)o->nq);
    for (int64_t j = 0; j < o->np; ++j) {
      ORC_PHASE(ORC_PH_PUSH_ION);
      o->AEA[j] = o->AEAN[j];
      o->AG[j] = o->AGN[j];
      push_particle(o, j);
    }
    ORC_PHASE(ORC_PH_MASTER);
    return;
  }
  int master = is_master(o, n);
  uint32_t nn = (uint32_t)(n / P->ndatfac + 1);
  if (master && o->pending) { /* ConvectionSub first, :62 */
    convection(o);
    free_tube(o->pending);
    o->pending = NULL;
  }
  if (master) /* Te update :69-89 */
    for (int Q = 0; Q < o->nq; ++Q)
      if (o->Te[Q] + P->dNTe <= P->dNTeEND)
        o->Te[Q] = o->Te[Q] + P->dNTe;
  ORC_PHASE(ORC_PH_CX);
  if (P->QEXCHANGEflag == 1)
    charge_exchange(o);
  ORC_PHASE(ORC_PH_MASTER);
  int64_t nexist = o->np;
  if (master) {
    o->lb_out = o->ub_out = o->lb_in = o->ub_in = 0;
    boundary(o);
    nexist = o->np;
    if (P->EAMBflag == 1)
      ambipolar(o, o->M0prev);
    gravfield(o);
    interpolate_particles(o, 0, NULL);
  }
  for (int64_t j = 0; j < nexist; ++j) {
    ORC_PHASE(o->ena[j] ? ORC_PH_PUSH_ENA : ORC_PH_PUSH_ION);
    if (!o->ena[j]) {
      o->AEA[j] = o->AEAN[j];
      o->AG[j] = o->AGN[j];
    }
    push_particle(o, j);
  }
  ORC_PHASE(ORC_PH_MASTER);
  if (master) {
    if (P->LBCONDITIONflag == 1)
      inject(o, 0);
    if (P->UBCONDITIONflag == 1)
      inject(o, 1);
    statistics(o);
    if (P->QEXCHANGEflag == 1) {
      collision_frequency(o, nn);
      ena_statistics(o);
    }
    memcpy(o->M0prev, o->mom[KAOS_M0], sizeof(double) * (size_t)o->nq);
    memcpy(o->mom[KAOS_EAMAG], o->EAmag, sizeof(double) * (size_t)o->nq);
    memcpy(o->mom[KAOS_EGMAG], o->EG, sizeof(double) * (size_t)o->nq);
  }
}

/* ======================================================================== */
/* exported API (mirrors include/kaos_gpu.h for the test harness)           */

orc *orc_create(const kaos_params_c *p, const kaos_tube_c *t,
                const kaos_vgrid_c *vg) {
  /* MomentFilterSub reads Pt cells around each cell: a tube shorter than a
   * window would read outside the arrays (the library rejects it too) */
  if (p->MOMENTFILTERflag == 1) {
    const int pts[5] = {p->M0MAfilterPt, p->M1ParMAfilterPt, p->M1Perp1MAfilterPt,
                        p->M1Perp2MAfilterPt, p->M2ParMAfilterPt};
    for (int k = 0; k < 5; ++k)
      if (pts[k] < 3 || pts[k] % 2 == 0 || t->nq < pts[k])
        return NULL;
  }
  orc *o = (orc *)calloc(1, sizeof(orc));
  o->P = *p;
  if (o->P.ndatfac < 1)
    o->P.ndatfac = 1;
  if (t->ms > 0.0) /* species of this entry (SpecieT(s)%msT, qsT) */
    o->P.ms = t->ms;
  if (t->qs != 0.0)
    o->P.qs = t->qs;
  int nq = t->nq;
  o->nq = nq;
  o->pG = t->pG;
  o->phiG = t->phiG;
  o->nsnormfac = t->nsnormfac;
  o->nsnormCLB = t->nsnormCLB;
  o->nsnormCUB = t->nsnormCUB;
  o->sumdsICR = t->sumdsICR;
#define D(a) o->a = dup(t->a, nq);
  D(qGL) D(qGH) D(qGC) D(hqC) D(dqC) D(d3xC) D(rGC) D(thetaGC) D(ellGC)
  D(TeG) D(TsG) D(nsnormCNeut) D(lambdaPerp) D(EtaLH) D(XiPerp1) D(XiPerp2)
  D(S0) D(OmegaG0) D(ChiPerp1) D(ChiPerp2)
#undef D
  o->n1 = vg->n1;
  o->n2 = vg->n2;
  o->npar = vg->npar;
  int d3 = p->ION2VPERPflag == 1;
  o->nv = d3 ? vg->n1 * vg->n2 * vg->npar : vg->n1 * vg->npar;
  o->e1 = dup(vg->e1, vg->n1 + 1);
  o->e2 = dup(vg->e2, d3 ? vg->n2 + 1 : 1);
  o->epar = dup(vg->epar, vg->npar + 1);
  o->c1 = dup(NULL, vg->n1);
  o->c2 = dup(NULL, d3 ? vg->n2 : 1);
  o->cpar = dup(NULL, vg->npar);
  for (int k = 0; k < vg->n1; ++k)
    o->c1[k] = (o->e1[k] + o->e1[k + 1]) / 2.0;
  for (int k = 0; d3 && k < vg->n2; ++k)
    o->c2[k] = (o->e2[k] + o->e2[k + 1]) / 2.0;
  for (int k = 0; k < vg->npar; ++k)
    o->cpar[k] = (o->epar[k] + o->epar[k + 1]) / 2.0;
  /* ENA grid: the ion grid's axes until orc_set_ena_grid (Vp <- Vperp1,
   * Vq <- Vpar, Vphi <- Vperp2, or Vperp1 on a 2D ion grid) */
  o->nep = vg->n1;
  o->eep = dup(vg->e1, vg->n1 + 1);
  o->neq = vg->npar;
  o->eeq = dup(vg->epar, vg->npar + 1);
  o->neph = d3 ? vg->n2 : vg->n1;
  o->eeph = d3 ? dup(vg->e2, vg->n2 + 1) : dup(vg->e1, vg->n1 + 1);
  o->d3v = dup(NULL, o->nv);
  for (int b = 0; b < o->nv; ++b) {
    double v;
    if (d3) {
      int i1 = b / (o->n2 * o->npar), i2 = (b / o->npar) % o->n2, ip = b % o->npar;
      v = 1.0 * 1.0 * 1.0 * fabs(o->e1[i1 + 1] - o->e1[i1]) *
          fabs(o->e2[i2 + 1] - o->e2[i2]) * fabs(o->epar[ip + 1] - o->epar[ip]);
    } else {
      int i1 = b / o->npar, ip = b % o->npar;
      v = 1.0 * 1.0 * fabs(o->c1[i1]) * fabs(o->e1[i1 + 1] - o->e1[i1]) *
          fabs(o->epar[ip + 1] - o->epar[ip]) * (2.0 * PI);
    }
    o->d3v[b] = (v == 0.0) ? 1e-9 : v;
  }
  o->Te = dup(t->TeG, nq);
  o->EAmag = dup(NULL, nq);
  o->EG = dup(NULL, nq);
  o->M0prev = dup(NULL, nq);
  o->nuPoi = dup(NULL, nq);
  o->EAimport = dup(NULL, nq);
  for (int k = 0; k < KAOS_NMOMENTS; ++k)
    o->mom[k] = dup(NULL, nq);
  o->cnt = (int64_t *)calloc((size_t)nq, sizeof(int64_t));
  o->hist = (int64_t *)calloc((size_t)nq * (size_t)o->nv, sizeof(int64_t));
  ensure_cap(o, 16);
  return o;
}

int orc_load(orc *o, const double *q, const double *vpar, const double *v1,
             const double *v2, int64_t n) {
  ensure_cap(o, n);
  o->np = n;
  double s = orient(o);
  for (int64_t j = 0; j < n; ++j) {
    double qq = q[j];
    /* KineticSolverA q clamp :55-65 (oriented) */
    if (s * qq <= s * o->qGL[0])
      qq = o->qGL[0];
    else if (s * qq > s * o->qGH[o->nq - 1])
      qq = o->qGH[o->nq - 1];
    o->id[j] = (uint64_t)j;
    place_ion(o, j, qq, vpar[j], v1[j], v2 ? v2[j] : 0.0);
  }
  o->next_id = (uint64_t)n;
  o->loaded = 1;
  return 0;
}

/* Initial-ion generator of kaos_init_particles (test input synthesis, the
 * same draws as the device generator): counts[k] ions in cell k, q uniform
 * over the middle 96 % of the cell, isotropic Maxwellian at TsG or, with
 * probability tail_fraction, an isotropic kappa distribution of temperature
 * tail_T drawn as a Student-t vector of nu = 2 kappa - 1 degrees of freedom
 * (covariance nu/(nu-2) s^2 = kT/m).  Philox (seed, ion index, 0,
 * KAOS_RNG_INIT << 24 | sub): sub 0 = (position, population) uniforms,
 * sub 1.. = Box-Muller pairs.  Then loaded as orc_load does. */
static void init_pair(uint64_t seed, uint64_t id, uint32_t sub, double *a,
                      double *b) {
  kaos_u32x4 w = kaos_philox((uint32_t)id, (uint32_t)(id >> 32), 0u,
                             (KAOS_RNG_INIT << 24) | sub, seed);
  double u1 = kaos_u01(w.v[0], w.v[1]), u2 = kaos_u01(w.v[2], w.v[3]);
  double R = sqrt(-2.0 * log(u1));
  *a = R * cos(2.0 * PI * u2);
  *b = R * sin(2.0 * PI * u2);
}

int orc_init(orc *o, const int64_t *counts, double tail_fraction, double kappa,
             double tail_T, uint64_t seed) {
  int64_t n = 0;
  for (int k = 0; k < o->nq; ++k)
    n += counts[k];
  double *q = (double *)malloc(sizeof(double) * (size_t)(n + 1));
  double *vp = (double *)malloc(sizeof(double) * (size_t)(n + 1));
  double *v1 = (double *)malloc(sizeof(double) * (size_t)(n + 1));
  double *v2 = (double *)malloc(sizeof(double) * (size_t)(n + 1));
  const int nu = (int)llround(2.0 * kappa - 1.0);
  const double st = sqrt(KB * tail_T / o->P.ms * (double)(nu - 2) / (double)nu);
  int64_t j = 0;
  for (int k = 0; k < o->nq; ++k)
    for (int64_t c = 0; c < counts[k]; ++c, ++j) {
      kaos_u32x4 w = kaos_philox((uint32_t)j, (uint32_t)((uint64_t)j >> 32), 0u,
                                 (KAOS_RNG_INIT << 24), seed);
      double upos = kaos_u01(w.v[0], w.v[1]), upop = kaos_u01(w.v[2], w.v[3]);
      q[j] = o->qGL[k] + (0.02 + 0.96 * upos) * (o->qGH[k] - o->qGL[k]);
      int tail = upop < tail_fraction;
      double g[66];
      int ng = 3 + (tail ? nu : 0);
      for (int m = 0; m < ng; m += 2)
        init_pair(seed, (uint64_t)j, (uint32_t)(1 + m / 2), &g[m], &g[m + 1]);
      double f;
      if (!tail) {
        f = sqrt(KB * o->TsG[k] / o->P.ms);
      } else {
        double W = 0.0;
        for (int m = 0; m < nu; ++m)
          W = W + g[3 + m] * g[3 + m];
        f = st / sqrt(W / (double)nu);
      }
      vp[j] = f * g[0];
      v1[j] = f * g[1];
      v2[j] = f * g[2];
    }
  int rc = orc_load(o, q, vp, v1, v2, n);
  free(q);
  free(vp);
  free(v1);
  free(v2);
  return rc;
}

int orc_set_fields(orc *o, const double *EA) {
  if (!EA) {
    o->have_import = 0;
    return 0;
  }
  memcpy(o->EAimport, EA, sizeof(double) * (size_t)o->nq);
  o->have_import = 1;
  return 0;
}

void orc_set_literal(orc *o, int on) { o->literal = on; }

/* A deep copy of a tube's tables, held until the next master step. */
static kaos_tube_c *copy_tube(const kaos_tube_c *t) {
  kaos_tube_c *c = (kaos_tube_c *)malloc(sizeof(kaos_tube_c));
  *c = *t;
  const double **f[] = {&c->qGL, &c->qGH, &c->qGC, &c->hqC, &c->dqC, &c->d3xC,
                        &c->rGC, &c->thetaGC, &c->ellGC, &c->TeG, &c->TsG,
                        &c->nsnormCNeut, &c->lambdaPerp, &c->EtaLH, &c->XiPerp1,
                        &c->XiPerp2, &c->S0, &c->OmegaG0, &c->ChiPerp1, &c->ChiPerp2};
  for (size_t k = 0; k < sizeof(f) / sizeof(f[0]); ++k)
    *f[k] = *f[k] ? dup(*f[k], t->nq) : NULL;
  return c;
}

static void free_tube(kaos_tube_c *c) {
  if (!c)
    return;
  const double *f[] = {c->qGL, c->qGH, c->qGC, c->hqC, c->dqC, c->d3xC, c->rGC,
                       c->thetaGC, c->ellGC, c->TeG, c->TsG, c->nsnormCNeut,
                       c->lambdaPerp, c->EtaLH, c->XiPerp1, c->XiPerp2, c->S0,
                       c->OmegaG0, c->ChiPerp1, c->ChiPerp2};
  for (size_t k = 0; k < sizeof(f) / sizeof(f[0]); ++k)
    free((void *)f[k]);
  free(c);
}

/* Test hook: apply a pending tube move now. */
void orc_convect_now(orc *o) {
  if (!o->pending)
    return;
  convection(o);
  free_tube(o->pending);
  o->pending = NULL;
}

/* ConvectionSub's tube move: applied at the next master step. */
int orc_update_tube(orc *o, const kaos_tube_c *t) {
  if (t->nq != o->nq)
    return 1;
  free_tube(o->pending);
  o->pending = copy_tube(t);
  return 0;
}

/* ENA velocity grid (Vp edges = e1/n1, Vphi = e2/n2, Vq = epar/npar). */
void orc_set_ena_grid(orc *o, const kaos_vgrid_c *vg) {
  free(o->eep);
  free(o->eeq);
  free(o->eeph);
  o->nep = vg->n1;
  o->eep = dup(vg->e1, vg->n1 + 1);
  o->neph = vg->n2;
  o->eeph = dup(vg->e2, vg->n2 + 1);
  o->neq = vg->npar;
  o->eeq = dup(vg->epar, vg->npar + 1);
}

int orc_step(orc *o, int64_t nsteps) {
  for (int64_t k = 0; k < nsteps; ++k)
    step_once(o);
  return 0;
}

int64_t orc_count(orc *o, int64_t *nena) {
  int64_t ni = 0, ne = 0;
  for (int64_t j = 0; j < o->np; ++j)
    if (o->ena[j])
      ne++;
    else
      ni++;
  if (nena)
    *nena = ne;
  return ni;
}

int orc_get_moments(orc *o, int which, double *out) {
  memcpy(out, o->mom[which], sizeof(double) * (size_t)o->nq);
  return 0;
}

int orc_get_counts(orc *o, int64_t *out, int64_t nbins) {
  if (nbins == o->nq)
    memcpy(out, o->cnt, sizeof(int64_t) * (size_t)o->nq);
  else
    memcpy(out, o->hist, sizeof(int64_t) * (size_t)o->nq * (size_t)o->nv);
  return 0;
}

/* ion state in reference order: q (from the stored Cartesian position),
 * Vpar (projection), Vperp1, Vperp2, Qindk1 (0-based, -1/-2 sentinels),
 * meridian-plane rho and z. */
int orc_get_particles(orc *o, double *q, double *vpar, double *v1, double *v2,
                      int32_t *qind, double *rho, double *zz) {
  int64_t k = 0;
  for (int64_t j = 0; j < o->np; ++j) {
    if (o->ena[j])
      continue;
    double r = sqrt(o->x[j] * o->x[j] + o->y[j] * o->y[j] + o->z[j] * o->z[j]);
    double th = acos(o->z[j] / r);
    double ct = cos(th), st = sin(th), cp = cos(o->phiG), sp = sin(o->phiG);
    double el = 1.0 + 3.0 * ct * ct;
    if (q)
      q[k] = (RE * RE) * ct / (r * r);
    if (vpar)
      vpar[k] = 3.0 * ct * st * (o->Vx[j] * cp + o->Vy[j] * sp) / sqrt(el) +
                o->Vz[j] * (3.0 * ct * ct - 1.0) / sqrt(el);
    if (v1)
      v1[k] = o->V1[j];
    if (v2)
      v2[k] = o->V2[j];
    if (qind) {
      int64_t Q = o->Qind[j];
      qind[k] = (int32_t)(Q >= 1 ? Q - 1 : (Q == 0 ? -1 : -2));
    }
    if (rho)
      rho[k] = o->x[j] * cp + o->y[j] * sp;
    if (zz)
      zz[k] = o->z[j];
    k++;
  }
  return 0;
}

int orc_get_enas(orc *o, double *x, double *y, double *z, double *vx,
                 double *vy, double *vz) {
  int64_t k = 0;
  for (int64_t j = 0; j < o->np; ++j) {
    if (!o->ena[j])
      continue;
    x[k] = o->x[j];
    y[k] = o->y[j];
    z[k] = o->z[j];
    vx[k] = o->Vx[j];
    vy[k] = o->Vy[j];
    vz[k] = o->Vz[j];
    k++;
  }
  return 0;
}

void orc_get_boundary(orc *o, int64_t *v) {
  v[0] = o->lb_out;
  v[1] = o->ub_out;
  v[2] = o->lb_in;
  v[3] = o->ub_in;
}

void orc_get_boundary_ena(orc *o, int64_t *v) {
  v[0] = o->lbe_out;
  v[1] = o->ube_out;
}

/* single quartic evaluation for known-answer tests */
/* The words of Philox4x32-10 (include/kaos_philox.h, the generator the
 * library and this checker share) for one counter and key: the hook of the
 * known-answer test against the published Random123 vectors. */
void orc_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                uint64_t key, uint32_t *out4) {
  kaos_u32x4 w = kaos_philox(c0, c1, c2, c3, key);
  for (int k = 0; k < 4; ++k) out4[k] = w.v[k];
}

void orc_quartic(double q, double p, double phi, double *out6) {
  double r, th, x, y, z;
  quartic(q, p, phi, &r, &th, &x, &y, &z);
  out6[0] = r;
  out6[1] = th;
  out6[2] = x;
  out6[3] = y;
  out6[4] = z;
  out6[5] = (RE * RE) * cos(th) / (r * r);
}

void orc_filter(const double *in, double *out, int nq, int pt) {
  moment_filter(in, out, nq, pt);
}

void orc_destroy(orc *o) {
  if (!o)
    return;
  double **ds[] = {&o->qGL, &o->qGH, &o->qGC, &o->hqC, &o->dqC, &o->d3xC,
                   &o->rGC, &o->thetaGC, &o->ellGC, &o->TeG, &o->TsG,
                   &o->nsnormCNeut, &o->lambdaPerp, &o->EtaLH, &o->XiPerp1,
                   &o->XiPerp2, &o->S0, &o->OmegaG0, &o->ChiPerp1,
                   &o->ChiPerp2, &o->e1, &o->e2, &o->epar, &o->c1, &o->c2,
                   &o->cpar, &o->d3v, &o->x, &o->y, &o->z, &o->Vx, &o->Vy,
                   &o->Vz, &o->V1, &o->V2, &o->Vp, &o->AEA, &o->AG, &o->AEAN,
                   &o->AGN, &o->qk4, &o->rk4, &o->thk4, &o->phk4, &o->ellk4,
                   &o->Vpe, &o->Vphe, &o->Te, &o->EAmag, &o->EG, &o->M0prev,
                   &o->nuPoi, &o->EAimport, &o->eep, &o->eeq, &o->eeph};
  for (size_t k = 0; k < sizeof(ds) / sizeof(ds[0]); ++k)
    free(*ds[k]);
  for (int k = 0; k < KAOS_NMOMENTS; ++k)
    free(o->mom[k]);
  free(o->Qind);
  free(o->ipar);
  free(o->i1);
  free(o->i2);
  free(o->iep);
  free(o->ieq);
  free(o->ieph);
  free(o->ena);
  free(o->id);
  free(o->cnt);
  free(o->hist);
  free_tube(o->pending);
  free(o);
}

/* test hook: the ambipolar pressure field of a given M0 profile (with the
 * tube's Te), as AmbipolarEfieldSub computes it on a master step. */
void orc_ambipolar(orc *o, const double *M0, double *EA) {
  ambipolar(o, M0);
  memcpy(EA, o->EAmag, sizeof(double) * (size_t)o->nq);
}

/* test hook: the Cartesian force at a point (KineticUpdateA) */
void orc_force(orc *o, double x, double y, double z, double Vperp, double AEA,
               double AG, double *out4) {
  fpoint f = force_ion(o, x, y, z, Vperp, AEA, AG);
  out4[0] = f.Ax;
  out4[1] = f.Ay;
  out4[2] = f.Az;
  out4[3] = f.q;
}
