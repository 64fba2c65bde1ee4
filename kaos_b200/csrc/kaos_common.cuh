// kaos_common.cuh -- device data layout and the per-point dipole geometry
// shared by the B200 kernels of the kinetic particle loop.
//
// Layout in HBM (one allocation per array, all tubes concatenated):
//  * ions: structure of arrays, tube t owns [tube.off, tube.off + tube.cap).
//    FP64 mode stores the meridian-plane position (rho, z) -- the ion motion
//    is confined to its flux-tube meridian (phi = phiG) -- plus V||, Vperp1,
//    Vperp2 and the cached field accelerations.  Mixed mode keeps its state
//    in FP64 accumulators and does its arithmetic in FP32: the position as
//    one FP64 cell coordinate (integer part = cell, fraction = offset in q
//    within the cell), V|| and the (Vperp1, Vperp2) pair in FP64, the
//    cached field accelerations (AEA, AG) and q_k4 in FP32.
//  * per-cell tables: concatenated over tubes, tube t at [tube.coff, +nq).
//  * velocity-grid edges: __constant__ memory (shared by all tubes).
#pragma once
#include <cstdint>

#include "../../include/kaos_gpu.h"
#include "../../include/kaos_philox.h"

namespace kaos {

// _ModelInput.f90:35-43
constexpr double PI = 3.14159265358979323846;
constexpr double KB = 138e-25;
constexpr double EPS0 = 8.854e-12;
constexpr double MDIP = 8.06e15;
constexpr double GG = 667e-13;
constexpr double ME = 598e22;
constexpr double RE = 638e4;

constexpr int MAXV = 128;          // max velocity cells per axis
constexpr int DEAD = -3;           // ion slot converted to an ENA
constexpr int BELOW = -1;          // reference Qind 0  (below LB)
constexpr int ABOVE = -2;          // reference Qind -1 (above UB)
// mixed mode: the cell coordinate of a slot marked DEAD (any value below
// XDEAD_LIM; a live or escaped ion's coordinate is never that far out)
constexpr double XDEAD = -1e30, XDEAD_LIM = -1e29;
// status bits; ST_TIMEOUT is reserved (no kernel here waits on another)
constexpr uint32_t ST_NAN = 1u, ST_CAP = 2u, ST_TIMEOUT = 4u;

struct VGridC {
  int n1, n2, npar, three_d;
  double e1[MAXV + 1], e2[MAXV + 1], epar[MAXV + 1];
  float f1[MAXV + 1], f2[MAXV + 1], fpar[MAXV + 1];
};

// One tube, device side.
struct TubeD {
  int nq, coff;            // cells, offset into per-cell tables
  int64_t off, cap;        // particle segment
  int64_t ecap, eoff;      // ENA segment
  double pG, phiG, cphi, sphi, sgn;  // sgn = +1 when q increases upward
  double nsnormfac, nsnormCLB, nsnormCUB, sumdsICR;
  int64_t moff;            // offset of this tube's marginal counters
  int64_t hoff;            // offset of this tube's full histogram
  double rhoLB, zLB, rhoUB, zUB;     // injection points (cell centres)
  double ms, qs;                     // species mass [kg] and charge [C]
};

// Per-cell tables (device pointers, concatenated over tubes).
struct CellTables {
  const double *qGL, *qGH, *qGC, *hqC, *dqC, *d3xC, *rGC, *thetaGC, *ellGC;
  const double *TeG, *TsG, *nsnormCNeut;
  const double *lambdaPerp, *EtaLH, *XiPerp1, *XiPerp2, *S0, *OmegaG0,
      *ChiPerp1, *ChiPerp2;
  const double *uL, *uH;  // quartic root u = r/RE at the cell edges
  const double *uM;       // ... and at the cell's midpoint in q
  const double *hK1, *hK2, *hc1, *hc2, *hiom0;  // wave-heating constants
  double *Te, *EAmag, *EG, *M0prev, *nuPoi;
  double *mom;            // [KAOS_NMOMENTS][ncell_total]
  int64_t ncell_total;
};

// Ion particle arrays.  vpar (V||, FP64) serves both modes; FP64 mode adds
// rho, z, v1, v2, aea, ag, qk4, mixed mode x, v12, ffl, fqk4.
struct Ions {
  double *rho, *z, *vpar, *v1, *v2, *aea, *ag, *qk4;  // FP64 mode (+ vpar)
  double *rho4, *z4;   // FP64 + charge exchange: the k4 point of the step
  // mixed mode: x = cell + offset in q within the cell (FP64; XDEAD marks
  // a dead slot), v12 = (Vperp1, Vperp2) in FP64, and in FP32 the pair read
  // together ffl = (AEA, AG) and q at the k4 point
  double *x;
  double2 *v12;
  float2 *ffl;
  float *fqk4;
  int32_t *qind;       // start-of-step cell Qindk1 (0-based, sentinels)
  int32_t *vb;         // 2D grid: stale (vperp,vpar) bins, packed
  uint64_t *id;        // persistent particle id (RNG key, order key)
};

struct Enas {
  double *x, *y, *z, *vx, *vy, *vz, *vps, *vphs;  // vps/vphs: stale Vp, Vphi
  int32_t *qind;
  int32_t *vb;   // Vp | Vq << 10 | Vphi << 20 bin indices, 1-based, 0: none
  uint64_t *id;
};

// Binning accumulators of one master step.
struct Accum {
  unsigned int *cnt;   // [ncell_total] ions with Qindk1 == cell
  unsigned int *m1, *m2, *mpar;  // marginals [cell][n]
  unsigned int *hist;  // optional full histogram [cell][nv]
  unsigned int *cxc;   // charge-exchange chunk counts
  // ENAs: per-cell counts and (Vp, Vq, Vphi) marginals [cell][MAXV]
  unsigned int *ecnt, *emp, *emq, *emph;
};

// ---- small helpers ------------------------------------------------------
// Warp sum (every lane gets the total).
__device__ __forceinline__ double warp_sum(double x) {
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// |Vperp| = sqrt(V1^2 + V2^2) with every product and the sum rounded on
// its own (no fused multiply-add): the value the 2D velocity-bin search
// compares, the same on every path and in the CPU oracle.
__device__ __forceinline__ double vperp_mag(double a, double b) {
  return sqrt(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)));
}

// Mixed mode: the cell of a cell coordinate x (clamped to the tube: an
// escaped ion keeps its end cell and an offset outside [0, 1]).
__device__ __forceinline__ int x_cell(double x, int nq) {
  return min(max(__double2int_rd(x), 0), nq - 1);
}

__host__ __device__ __forceinline__ int64_t ceil_div(int64_t a, int64_t b) {
  return (a + b - 1) / b;
}

// Oriented cell search over contiguous edges E[0..nq] (oriented so they
// increase): first cell [E0,E1], later cells (Ek, Ek+1]; below -> BELOW,
// above -> ABOVE (KineticUpdateA _8_1_1_KineticUpdateA.f90:221-273).
__device__ __forceinline__ int cell_search(const double *E, int nq, double s) {
  if (s < E[0]) return BELOW;
  if (s > E[nq]) return ABOVE;
  int lo = 1, hi = nq;  // smallest k in [1,nq] with s <= E[k]
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (s <= E[mid]) hi = mid; else lo = mid + 1;
  }
  return lo - 1;
}

// Velocity-bin search (:994-1129): smallest k>=1 with v <= e[k] gives bin
// k-1; first bin closed.  Out of range -> -1.
template <typename T>
__device__ __forceinline__ int vbin(const T *e, int n, T v) {
  if (!(v >= e[0] && v <= e[n])) return -1;
  int lo = 1, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (v <= e[mid]) hi = mid; else lo = mid + 1;
  }
  return lo - 1;
}

// Dipole geometry at a meridian-plane point and the field-aligned
// acceleration (KineticUpdateA/B/C force blocks, _KineticMainParams.f90:
// 568-804).  Every force term is parallel to the unit vector e along B, so
// the Cartesian sums of the reference reduce to a scalar a|| times e.
template <typename T> struct Geo {
  T ct, st, ir, q, isl, ell, er, ez;  // cos, sin, 1/r, q, 1/sqrt(ell), ell, e
};

__device__ __forceinline__ double rsq(double x) { return rsqrt(x); }
// FP32: one MUFU operation, denormals flushed (the FP32 geometry of the
// mixed push never comes near the denormal range).
__device__ __forceinline__ float rsq(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

template <typename T>
__device__ __forceinline__ Geo<T> geo(T rho, T z) {
  Geo<T> g;
  T r2 = rho * rho + z * z;
  T ir = rsq(r2);
  g.ir = ir;
  g.ct = z * ir;
  g.st = rho * ir;
  g.q = T(RE * RE) * g.ct * (ir * ir);
  g.ell = T(1) + T(3) * g.ct * g.ct;
  g.isl = rsq(g.ell);
  g.er = T(3) * g.ct * g.st * g.isl;
  g.ez = (T(3) * g.ct * g.ct - T(1)) * g.isl;
  return g;
}

struct ForceFlags {
  int mirror, grav, eamb, eambsign;
};

// a|| = mirror + gravity + ambipolar at the point described by g.
//  mirror: -mu dB/ds / ms with mu = ms Vperp^2/(2B), sign from hemisphere
//  gravity: -+|AG| (toward the Earth), ambipolar: AEA (EAMBSIGN=1).
template <typename T>
__device__ __forceinline__ T apar(const Geo<T> &g, T vperp2, T aea, T ag,
                                  ForceFlags f) {
  T a = T(0);
  bool south = (g.ct <= T(0));  // the sign of q = RE^2 cos(theta) / r^2
  if (f.mirror) {
    // |mu dBds/ms| = Vperp^2/2 * 3 ct/r (2 + st^2/ell)/sqrt(ell)
    T m = T(1.5) * vperp2 * fabs(g.ct) * g.ir * (T(2) + g.st * g.st * g.isl * g.isl) * g.isl;
    a += south ? -m : m;
  }
  if (f.grav) a += south ? fabs(ag) : -fabs(ag);
  if (f.eamb) {
    if (f.eambsign) a += aea;
    else a += south ? -fabs(aea) : fabs(aea);
  }
  return a;
}

}  // namespace kaos
