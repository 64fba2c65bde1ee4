// kaos_cx.cuh -- ion -> ENA charge exchange and the ballistic ENA push.
//
// Reference: the production loop of KineticSolverSub
// (_8_KineticSolver.f90:95-166) converts, on every computational step, the
// first nint(nuIonNeutPoiT(nn-1,Q)) ions (in particle-index order) whose
// Qindk1 is Q into ENAs (IonNeutralCollisionsSub
// _8_1_1_1_IonNeutralCollisions.f90:25-58); ENAs then move under gravity
// only (AGENA*sub _KineticMainParams.f90:695-714, KineticRK4UpdateSub
// :186-193, :292-314).
//
// Selection on the GPU keeps the index order exactly: the push that writes
// Qindk1 also counts, per selection chunk of CX_CHUNK ions, the ions of each
// cell (flush_cx_counts); a scan over chunks per cell follows (what each
// chunk still owes each cell, and the list of chunks that convert), then a
// parallel selection of the first owed ions per cell in each listed chunk,
// equal to a walk in index order.
#pragma once
#include "kaos_push.cuh"

namespace kaos {

constexpr int CX_CHUNK = 16384;  // particles per selection chunk

struct CxArgs {
  const TubeD *tubes;
  const int *cx_tube;        // chunk -> tube
  const int64_t *cx_start;   // chunk -> first particle (tube-relative)
  const int *tube_cx0;       // first chunk of each tube (ntubes+1)
  const int64_t *nlive;
  CellTables ct;
  Ions ion;
  Enas ena;
  int64_t *nena;
  unsigned *cxc;             // [chunk][nq_max] Qindk1 counts (from the push)
  unsigned *cxo;             // [chunk][nq_max] conversions still owed there
  unsigned *cxconv;          // per chunk: ions converted in it this step
  int64_t *cxbase;           // per chunk: ENA slot of its first conversion
  int *cxend;                // per cell (all tubes): chunks >= cxend convert none
  int *tube_done;            // per tube: cell scans finished this step
  int *list, *nlist;         // cells with conversions (need > 0), their count
  // chunks with conversions this step, appended by the scan; [0] their
  // count, [1] conversion blocks that have read it (the last one resets
  // both for the next step)
  int *chunk_list;
  unsigned *nchunk;
  int *tube_active;          // per tube: listed cells
  int nqmax, mixed;
  int ncx;                   // selection chunks (all tubes)
  int rank, nranks;          // this rank's share of a split tube's conversions
  uint32_t *status;
};

// Ions a cell converts at this step on this rank: its share of
// nint(nuIonNeutPoiT) when the tube is split over nranks.
__device__ __forceinline__ unsigned cx_need(const CxArgs &a, double nu) {
  const unsigned n = nu > 0.0 ? (unsigned)llrint(nu) : 0u;
  return a.nranks > 1 ? (n + (unsigned)a.rank) / (unsigned)a.nranks : n;
}

// exclusive scan over the chunks of a tube for one cell (one block per
// (tube, cell) pair, block-wide scan, blockDim.x chunks a pass); adds the conversions of this cell to
// the per-chunk totals.
// A cell with no conversion does nothing; the scan of a cell stops after the
// tile of chunks in which its prefix reaches the conversion count, and
// cxend records the first chunk without a written prefix.  Only the chunks
// holding live ions are scanned: the push writes no count beyond them.
__device__ __forceinline__ int cx_live_end(const CxArgs &a, int t) {
  const int c0 = a.tube_cx0[t], c1 = a.tube_cx0[t + 1];
  return (int)min((int64_t)c1, c0 + ceil_div(a.nlive[t], (int64_t)CX_CHUNK));
}

__device__ __forceinline__ void cx_scan_cell(const CxArgs &a, int t, int k,
                                             int g) {
  const TubeD &T = a.tubes[t];
  const unsigned need = cx_need(a, a.ct.nuPoi[T.coff + k]);
  if (need == 0u) return;
  const int c0 = a.tube_cx0[t], c1 = cx_live_end(a, t);
  __shared__ unsigned wsum[32];
  __shared__ unsigned base;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  const int l = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int r0 = c0; r0 < c1; r0 += blockDim.x) {
    const int c = r0 + threadIdx.x;
    const unsigned n = (c < c1) ? a.cxc[(int64_t)c * a.nqmax + k] : 0u;
    unsigned x = n;  // inclusive warp scan
    for (int o = 1; o < 32; o <<= 1) {
      unsigned y = __shfl_up_sync(0xffffffffu, x, o);
      if (l >= o) x += y;
    }
    if (l == 31) wsum[w] = x;
    __syncthreads();
    unsigned woff = 0, tot = 0;
    for (int v = 0; v < nw; ++v) { if (v < w) woff += wsum[v]; tot += wsum[v]; }
    const unsigned s = base + woff + x - n;  // exclusive prefix
    if (c < c1) {
      a.cxo[(int64_t)c * a.nqmax + k] = s < need ? need - s : 0u;
      // the first cell to give the chunk a conversion lists it
      if (n && s < need && atomicAdd(&a.cxconv[c], min(n, need - s)) == 0u)
        a.chunk_list[atomicAdd(a.nchunk, 1u)] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) base += tot;
    __syncthreads();
    if (base >= need) {
      if (threadIdx.x == 0) a.cxend[g] = min(r0 + (int)blockDim.x, c1);
      return;
    }
  }
  if (threadIdx.x == 0) a.cxend[g] = c1;
}

// ENA slots in ion-index order: exclusive scan of the per-chunk conversion
// totals over the live chunks of each tube (one block per tube, each thread
// a run of consecutive chunks: run sums, one block scan, run prefixes); the
// ENA count of the tube advances by the step's total.
__device__ __forceinline__ void cx_base_tube(const CxArgs &a, int t) {
  const int c0 = a.tube_cx0[t], c1 = cx_live_end(a, t);
  __shared__ unsigned long long wsum[32];
  const int64_t n0 = a.nena[t];
  const int l = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int run = (int)ceil_div((int64_t)max(c1 - c0, 0), (int64_t)blockDim.x);
  const int r0 = c0 + (int)threadIdx.x * run, r1 = min(r0 + run, c1);
  unsigned long long n = 0;  // (L2 reads: other blocks' atomics)
  for (int c = r0; c < r1; ++c) n += __ldcg(a.cxconv + c);
  unsigned long long x = n;  // inclusive warp scan of the run sums
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (l >= o) x += y;
  }
  if (l == 31) wsum[w] = x;
  __syncthreads();
  unsigned long long woff = 0, tot = 0;
  for (int v = 0; v < nw; ++v) { if (v < w) woff += wsum[v]; tot += wsum[v]; }
  unsigned long long s = woff + x - n;  // exclusive prefix of this run
  for (int c = r0; c < r1; ++c) {
    a.cxbase[c] = n0 + (int64_t)s;
    s += __ldcg(a.cxconv + c);
  }
  if (threadIdx.x == 0) a.nena[t] = n0 + (int64_t)tot;
}

// The cells that convert ions (need > 0) are listed once per master step,
// when the collision counts change, with each tube's number of them.
__global__ void k_cx_list(CxArgs a, const int *cell_tube, int64_t ncell) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ncell) return;
  a.cxend[g] = 0;  // a cell off the list owes nothing in any chunk
  if (cx_need(a, a.ct.nuPoi[g]) == 0u) return;
  a.list[atomicAdd(a.nlist, 1)] = (int)g;
  atomicAdd(a.tube_active + cell_tube[g], 1);
}

// A block (256 threads) per listed cell, striding over the list: the cell's
// scan, then the last listed cell of a tube to finish (a per-tube arrival
// counter) gives the tube its ENA slots and resets the counter.
// Tubes without a listed cell convert nothing this step.
__global__ void __launch_bounds__(256) k_cx_scan(CxArgs a, const int *cell_tube,
                                                  const int *cell_q) {
  const int nl = *a.nlist;
  __shared__ int last;
  for (int i = blockIdx.x; i < nl; i += gridDim.x) {
    const int g = a.list[i];
    const int t = cell_tube[g], k = cell_q[g];
    __syncthreads();  // the previous cell of this block is done with smem
    cx_scan_cell(a, t, k, g);
    __syncthreads();  // every thread's counts and prefixes are written
    if (threadIdx.x == 0) {
      __threadfence();
      last = atomicAdd(a.tube_done + t, 1) == a.tube_active[t] - 1;
      if (last) a.tube_done[t] = 0;
    }
    __syncthreads();
    if (last) {
      __threadfence();
      cx_base_tube(a, t);
    }
  }
}

// Cartesian unit vectors along B (par), across the shell (p) and in
// longitude (phi) at polar cos/sin (ct, st) and longitude (cp, sp).
__device__ __forceinline__ void dipole_frame(double ct, double st, double cp,
                                             double sp, double e_par[3],
                                             double e_p[3], double e_phi[3]) {
  const double isl = rsqrt(1.0 + 3.0 * ct * ct);
  const double a = 3.0 * ct * st * isl, b = (3.0 * ct * ct - 1.0) * isl;
  const double c = (1.0 - 3.0 * ct * ct) * isl;
  e_par[0] = cp * a; e_par[1] = sp * a; e_par[2] = b;
  e_p[0] = cp * c;   e_p[1] = sp * c;   e_p[2] = a;
  e_phi[0] = -sp;    e_phi[1] = cp;     e_phi[2] = 0.0;
}

// The first item at or after `first` that belongs to this block of a grid
// striding over work items (item = blockIdx.x mod gridDim.x).
__device__ __forceinline__ int next_own_item(int first) {
  const int G = (int)gridDim.x;
  return first + (((int)blockIdx.x - first) % G + G) % G;
}

// Convert ion j (cell q) into the ENA of slot `slot`: the ion's state at the
// end of the previous step, its velocity rotated into the frame of the
// previous step's k4 point (IonNeutralCollisionsSub
// _8_1_1_1_IonNeutralCollisions.f90:25-58); the ion slot is marked DEAD.
__device__ __forceinline__ void cx_convert_ion(const CxArgs &a, const TubeD &T,
                                               int64_t j, int q, int64_t slot) {
  // ion position and velocity at the end of the previous step
  double rho, z, vpar, v1, v2, qk4;
  if (a.mixed) {
    const double xx = a.ion.x[j];
    const int cc = x_cell(xx, T.nq);
    const double oo = xx - (double)cc;
    const double qq = a.ct.qGL[T.coff + cc] +
                      oo * (a.ct.qGH[T.coff + cc] - a.ct.qGL[T.coff + cc]);
    const double ug = a.ct.uL[T.coff + cc] +
                      oo * (a.ct.uH[T.coff + cc] - a.ct.uL[T.coff + cc]);
    const double u = quartic_newton(qq, 1.0 / T.pG, ug, 3);
    const double s2 = u / T.pG;
    rho = u * RE * sqrt(s2);
    z = u * RE * qq * u * u;
    vpar = a.ion.vpar[j];
    const double2 v = a.ion.v12[j];
    v1 = v.x;
    v2 = v.y;
    qk4 = a.ion.fqk4[j];
  } else {
    rho = a.ion.rho[j];
    z = a.ion.z[j];
    vpar = a.ion.vpar[j];
    v1 = a.ion.v1[j];
    v2 = a.ion.v2[j];
    qk4 = a.ion.qk4[j];
  }
  // geometry of the k4 point of the previous step: stored exactly in
  // FP64 mode, rebuilt from its q (p = pG) in mixed mode
  double ctk, stk;
  if (a.ion.rho4) {
    const Geo<double> g4 = geo(a.ion.rho4[j], a.ion.z4[j]);
    ctk = g4.ct;
    stk = g4.st;
  } else {
    const double uk = quartic_newton(qk4, 1.0 / T.pG, sqrt(rho * rho + z * z) / RE, 4);
    ctk = qk4 * uk * uk;
    stk = sqrt(uk / T.pG);
  }
  const Geo<double> gN = geo(rho, z);
  double ep[3], epp[3], eph[3], e4[3], e4p[3], e4h[3];
  dipole_frame(gN.ct, gN.st, T.cphi, T.sphi, ep, epp, eph);
  dipole_frame(ctk, stk, T.cphi, T.sphi, e4, e4p, e4h);
  const double VN[3] = {vpar * ep[0], vpar * ep[1], vpar * ep[2]};
  const double vp4 = e4[0] * VN[0] + e4[1] * VN[1] + e4[2] * VN[2];
  if (slot < T.ecap) {
    const int64_t e = T.eoff + slot;
    a.ena.x[e] = rho * T.cphi;
    a.ena.y[e] = rho * T.sphi;
    a.ena.z[e] = z;
    a.ena.vx[e] = vp4 * e4[0] + v1 * e4p[0] + v2 * e4h[0];
    a.ena.vy[e] = vp4 * e4[1] + v1 * e4p[1] + v2 * e4h[1];
    a.ena.vz[e] = vp4 * e4[2] + v1 * e4p[2] + v2 * e4h[2];
    a.ena.vps[e] = 0.0;  // Vp(j), Vphi(j) still hold the ion zeros
    a.ena.vphs[e] = 0.0;
    a.ena.qind[e] = q;
    a.ena.vb[e] = 0;
    a.ena.id[e] = a.ion.id[j];
  } else {
    atomicOr(a.status, ST_CAP);
  }
  a.ion.qind[j] = DEAD;
  if (a.mixed) a.ion.x[j] = XDEAD;
}

// In-order conversion of the first need[Q] eligible ions per cell of one
// chunk, selected in parallel: each of the CX_WARPS warps owns a segment of
// CX_CHUNK / CX_WARPS consecutive ions.  Pass 1 counts every warp's
// candidates per cell; the counts become per-cell exclusive prefixes over
// the warps; pass 2 ranks each candidate among its cell's candidates of the
// chunk (prefix + running count in the segment), and rank < need converts
// -- the same ions as a walk in index order.  Each warp lists its
// conversions in order; they take consecutive ENA slots from cxbase in index
// order and are converted by all threads at once.
constexpr int CX_WARPS = 8;  // 256-thread blocks
static_assert(CX_CHUNK <= (1 << 14), "conversion list packs (cell << 14) | index");
__device__ __forceinline__ void cx_convert_chunk(const CxArgs &a, int c, int t) {
  // a copy: every barrier below would otherwise reload the fields from
  // global memory, and the staging traffic evicts them from L1
  const TubeD T = a.tubes[t];
  __syncthreads();  // the previous chunk of this block is done with smem
  extern __shared__ unsigned sm_[];
  unsigned *need = sm_;             // conversions this chunk owes per cell
  unsigned *wcnt = sm_ + a.nqmax;   // [CX_WARPS][nq]: counts, then ranks
  int *qs = (int *)(wcnt + CX_WARPS * a.nqmax);  // Qindk1, then the lists
  __shared__ unsigned wconv[CX_WARPS];
  const int64_t beg = a.cx_start[c];
  const int nk = (int)min((int64_t)CX_CHUNK, a.nlive[t] - beg);
  // owed by this chunk: written by this step's scan for the chunks before
  // the cell's cxend (0 off the list)
  for (int k = threadIdx.x; k < T.nq; k += blockDim.x) {
    const int ce = a.cxend[T.coff + k];
    const unsigned o = a.cxo[(int64_t)c * a.nqmax + k];
    need[k] = c < ce ? o : 0u;
  }
  for (int k = threadIdx.x; k < CX_WARPS * T.nq; k += blockDim.x) wcnt[k] = 0u;
  if (threadIdx.x == 0) a.cxconv[c] = 0u;  // for the next step's scan
  __syncthreads();
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  const unsigned lt = (1u << l) - 1u;
  constexpr int SEG = CX_CHUNK / CX_WARPS;  // ions per warp
  constexpr int GPW = SEG / 32;             // 32-ion groups per warp
  constexpr int BATCH = 16;                 // loads in flight per lane
  static_assert(GPW % 32 == 0 && GPW % BATCH == 0, "segment layout");
  __shared__ unsigned gmask[CX_WARPS * GPW];  // candidate lanes per group
  const int s0 = w * SEG, s1 = min(s0 + SEG, nk);
  // each warp stages its own segment: candidates (a cell that still
  // converts here) keep their cell, others -1; BATCH independent loads per
  // lane are issued before any is used
  const int32_t *qsrc = a.ion.qind + T.off + beg;
  if ((((uintptr_t)qsrc) & 15) == 0 && s1 == s0 + SEG) {
    // a full, 16-byte aligned segment: SEG / 128 int4 loads per lane, in
    // two batches of independent loads
    constexpr int NV = SEG / 256;
#pragma unroll
    for (int b = 0; b < 2; ++b) {
    int4 v[NV];
#pragma unroll
    for (int u = 0; u < NV; ++u)
      v[u] = *(const int4 *)(qsrc + s0 + 4 * ((b * NV + u) * 32 + l));
#pragma unroll
    for (int u = 0; u < NV; ++u) {
      int4 r;
      r.x = (v[u].x >= 0 && need[v[u].x] != 0u) ? v[u].x : -1;
      r.y = (v[u].y >= 0 && need[v[u].y] != 0u) ? v[u].y : -1;
      r.z = (v[u].z >= 0 && need[v[u].z] != 0u) ? v[u].z : -1;
      r.w = (v[u].w >= 0 && need[v[u].w] != 0u) ? v[u].w : -1;
      *(int4 *)(qs + s0 + 4 * ((b * NV + u) * 32 + l)) = r;
    }
    }
  } else {
    for (int g0 = 0; g0 < GPW; g0 += BATCH) {
      int v[BATCH];
#pragma unroll
      for (int u = 0; u < BATCH; ++u) {
        const int i = s0 + (g0 + u) * 32 + l;
        v[u] = i < s1 ? qsrc[i] : -1;
      }
#pragma unroll
      for (int u = 0; u < BATCH; ++u)
        qs[s0 + (g0 + u) * 32 + l] = (v[u] >= 0 && need[v[u]] != 0u) ? v[u] : -1;
    }
  }
  __syncwarp();
  for (int g = 0; g < GPW; ++g) {
    const unsigned m = __ballot_sync(0xffffffffu, qs[s0 + g * 32 + l] >= 0);
    if (l == 0) gmask[w * GPW + g] = m;
  }
  __syncwarp();
  unsigned *wc = wcnt + w * T.nq;
  // pass 1: this warp's candidates per cell (one leader per cell adds),
  // over the groups holding candidates only
  for (int h = 0; h < GPW; h += 32) {
    unsigned has = __ballot_sync(0xffffffffu, gmask[w * GPW + h + l] != 0u);
    while (has) {
      const int i = s0 + (h + __ffs(has) - 1) * 32 + l;
      has &= has - 1u;
      const int q = qs[i];
      const unsigned peers = __match_any_sync(0xffffffffu, q);
      if (q >= 0 && (peers & lt) == 0u) wc[q] += __popc(peers);
      __syncwarp();
    }
  }
  __syncthreads();
  // per cell: the counts become exclusive prefixes over the warps
  for (int k = threadIdx.x; k < T.nq; k += blockDim.x) {
    unsigned sum = 0;
    for (int v = 0; v < CX_WARPS; ++v) {
      const unsigned x = wcnt[v * T.nq + k];
      wcnt[v * T.nq + k] = sum;
      sum += x;
    }
  }
  __syncthreads();
  // pass 2: ranks; the k-th conversion of the segment is listed at qs[s0 +
  // k], at or before the entries of its own (already read) group, as
  // (cell << 14) | index
  unsigned nwc = 0;
  for (int h = 0; h < GPW; h += 32) {
    unsigned has = __ballot_sync(0xffffffffu, gmask[w * GPW + h + l] != 0u);
    while (has) {
      const int i = s0 + (h + __ffs(has) - 1) * 32 + l;
      has &= has - 1u;
      const int q = qs[i];
      const unsigned peers = __match_any_sync(0xffffffffu, q);
      const bool conv = q >= 0 && wc[q] + __popc(peers & lt) < need[q];
      __syncwarp();  // every lane has read its cell's running rank and entry
      if (q >= 0 && (peers & lt) == 0u) wc[q] += __popc(peers);
      const unsigned bal = __ballot_sync(0xffffffffu, conv);
      if (conv) qs[s0 + nwc + __popc(bal & lt)] = (q << 14) | i;
      nwc += __popc(bal);
      __syncwarp();
    }
  }
  if (l == 0) wconv[w] = nwc;
  __syncthreads();
  unsigned tot = 0;
  for (int v = 0; v < CX_WARPS; ++v) tot += wconv[v];
  const int64_t slot0 = a.cxbase[c];
  for (int m = threadIdx.x; m < (int)tot; m += blockDim.x) {
    int v = 0;
    unsigned off = 0;
    while (m >= (int)(off + wconv[v])) off += wconv[v++];
    const int e = qs[v * SEG + (m - (int)off)];
    cx_convert_ion(a, T, T.off + beg + (e & ((1 << 14) - 1)), e >> 14, slot0 + m);
  }
}

// One resident wave of blocks; each chunk the scan listed is converted by
// one block.
__global__ void __launch_bounds__(256, 2) k_cx_convert(CxArgs a) {
  __shared__ int nc_s;
  if (threadIdx.x == 0) {
    nc_s = (int)__ldcg(a.nchunk);
    __threadfence();
    if (atomicAdd(a.nchunk + 1, 1u) == gridDim.x - 1) {  // every block has read it
      a.nchunk[0] = 0u;
      a.nchunk[1] = 0u;
    }
  }
  __syncthreads();
  const int nc = nc_s;
  for (int k = blockIdx.x; k < nc; k += gridDim.x) {
    const int c = a.chunk_list[k];
    cx_convert_chunk(a, c, a.cx_tube[c]);
  }
}

// ---------------------------------------------------------------------------
// Ballistic ENA step under gravity (FP64): the ENA branch of
// KineticUpdateA/B/C and KineticRK4UpdateSub, including the reference's
// |Vp| in the rebuilt velocity (_8_1_1_KineticUpdateA.f90:1155-1160,
// _8_1_KineticRK4Update.f90:292-314) and the cell index for removal.
struct EnaArgs {
  const TubeD *tubes;
  const int *blk_tube;
  const int64_t *blk_start;
  const int *tube_blk0;  // first work item of each tube (ntubes + 1)
  int nitems;            // work items (tube, chunk of ENA slots)
  int chunk;
  int sub;               // units per item (a unit: chunk / sub slots, a block's)
  int ntubes, ct_nqmax;  // tubes; cells of the largest (shared-memory layout)
  const int64_t *nena;
  CellTables ct;
  Enas ena;
  Accum acc;
  double h, grav_GM;
  int grav;
  int bin;  // master step: count the ENAs by start-of-step cell and bins
};

// ENA velocity grid (V3CellT): n1/e1 = Vp, npar/epar = Vq, n2/e2 = Vphi.
__constant__ VGridC c_evg;

// ENA velocity-bin search (KineticUpdateA _8_1_1_KineticUpdateA.f90:1161-
// 1230), 1-based; the reference's out-of-grid test can never hold, so a
// value outside the grid keeps the previous index.
__device__ __forceinline__ int ena_bin(const double *e, int n, double v,
                                       int prev) {
  const int b = vbin(e, n, v);
  return b >= 0 ? b + 1 : prev;
}

__device__ __forceinline__ void ena_geo(const double x[3], double &ct,
                                        double &st, double &cp, double &sp,
                                        double &q, double &ir) {
  const double rho2 = x[0] * x[0] + x[1] * x[1];
  const double r2 = rho2 + x[2] * x[2];
  ir = rsqrt(r2);
  ct = x[2] * ir;
  const double rho = sqrt(rho2);
  st = rho * ir;
  if (rho > 0.0) { cp = x[0] / rho; sp = x[1] / rho; } else { cp = 1.0; sp = 0.0; }
  q = (RE * RE) * ct * ir * ir;
}

__device__ __forceinline__ void ena_acc(const EnaArgs &a, const double x[3],
                                        double A[3]) {
  if (!a.grav) { A[0] = A[1] = A[2] = 0.0; return; }
  const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
  const double ir = rsqrt(r2);
  const double g = -a.grav_GM * ir * ir * ir;
  A[0] = g * x[0]; A[1] = g * x[1]; A[2] = g * x[2];
}

// First unit of each tube (UP[0..ntubes], an exclusive prefix of the units
// holding ENAs this step): each thread a run of consecutive tubes, then one
// block-wide scan.
__device__ __forceinline__ void ena_unit_prefix(const EnaArgs &a, int *UP, int usz) {
  const int n = a.ntubes;
  const int run = (n + (int)blockDim.x - 1) / (int)blockDim.x;
  const int r0 = (int)threadIdx.x * run, r1 = min(r0 + run, n);
  int cnt = 0;
  for (int t = r0; t < r1; ++t) {
    const int64_t nl = min(a.nena[t], a.tubes[t].ecap);
    UP[t] = (int)ceil_div(nl, (int64_t)usz);
    cnt += UP[t];
  }
  __shared__ int wsum[32];
  const int l = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int x = cnt;  // inclusive warp scan of the run counts
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (l >= o) x += y;
  }
  if (l == 31) wsum[w] = x;
  __syncthreads();
  int off = x - cnt;
  for (int v = 0; v < w; ++v) off += wsum[v];
  for (int t = r0; t < r1; ++t) {
    const int c = UP[t];
    UP[t] = off;
    off += c;
  }
  if (threadIdx.x == blockDim.x - 1) UP[n] = off;
  __syncthreads();
}

// A grid striding over the units holding ENAs (one ENA per thread), found
// through the per-tube unit prefix; a unit's tube by binary search.
__global__ void __launch_bounds__(256, 3) k_push_ena(EnaArgs a) {
  extern __shared__ double sm[];
  double *E = sm;
  int *UP = (int *)(sm + a.ct_nqmax + 1);
  // the ENA grid's edges for the bin searches in shared memory (threads
  // read different edges: constant memory would serialise them)
  __shared__ double EE1[MAXV + 1], EE2[MAXV + 1], EEP[MAXV + 1];
  const double h = a.h, hh = 0.5 * h, h6 = h / 6.0, hsq2 = 0.5 * h * h;
  int tcur = -1;
  const int usz = a.chunk / a.sub;
  ena_unit_prefix(a, UP, usz);
  const int nunits = UP[a.ntubes];
  if ((int)blockIdx.x >= nunits) return;  // no unit for this block (uniform)
  load_vgrid_smem(c_evg.e1, c_evg.e2, c_evg.epar, EE1, EE2, EEP);
  __syncthreads();
  for (int unit = blockIdx.x; unit < nunits; unit += gridDim.x) {
  int lo = 0, hi = a.ntubes;  // UP[lo] <= unit < UP[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (UP[mid] <= unit) lo = mid; else hi = mid;
  }
  const int t = lo;
  // the tube's fields in registers: not reloaded after the barriers
  struct { int nq; double sgn; int64_t coff, eoff; } T;
  {
    const TubeD &G = a.tubes[t];
    T.nq = G.nq;
    T.sgn = G.sgn;
    T.coff = G.coff;
    T.eoff = G.eoff;
  }
  const int64_t nl = min(a.nena[t], a.tubes[t].ecap);
  const int64_t beg = (int64_t)(unit - UP[t]) * usz;
  const int64_t end = min(beg + (int64_t)usz, nl);
  if (t != tcur) {
    __syncthreads();  // the previous tube's edges are no longer read
    for (int k = threadIdx.x; k <= T.nq; k += blockDim.x)
      E[k] = (k < T.nq) ? T.sgn * a.ct.qGL[T.coff + k] : T.sgn * a.ct.qGH[T.coff + T.nq - 1];
    __syncthreads();
    tcur = t;
  }
  for (int64_t i = beg + threadIdx.x; i < end; i += blockDim.x) {
    const int64_t e = T.eoff + i;
    double x[3] = {a.ena.x[e], a.ena.y[e], a.ena.z[e]};
    const double V[3] = {a.ena.vx[e], a.ena.vy[e], a.ena.vz[e]};
    double ct, st, cp, sp, q, ir;
    ena_geo(x, ct, st, cp, sp, q, ir);
    int qi = cell_search(E, T.nq, T.sgn * q);
    double ep[3], epp[3], eph[3];
    dipole_frame(ct, st, cp, sp, ep, epp, eph);
    const double vpar = ep[0] * V[0] + ep[1] * V[1] + ep[2] * V[2];
    double vps = a.ena.vps[e], vphs = a.ena.vphs[e];
    const int vb = a.ena.vb[e];
    int ip = vb & 1023, iq = (vb >> 10) & 1023, iph = (vb >> 20) & 1023;
    if (qi >= 0) {
      vps = fabs(epp[0] * V[0] + epp[1] * V[1] + epp[2] * V[2]);
      vphs = eph[0] * V[0] + eph[1] * V[1];
      ip = ena_bin(EE1, c_evg.n1, vps, ip);
      iq = ena_bin(EEP, c_evg.npar, vpar, iq);
      iph = ena_bin(EE2, c_evg.n2, vphs, iph);
      const int nvb = ip | (iq << 10) | (iph << 20);
      if (nvb != vb) a.ena.vb[e] = nvb;
      // ENAParticleCountsSub (_8_3_2_ENAParticleCounts.f90:45-300)
      if (a.bin) {
        const int64_t gc = T.coff + qi;
        atomicAdd(a.acc.ecnt + gc, 1u);
        if (ip && iq && iph) {
          atomicAdd(a.acc.emp + gc * MAXV + (ip - 1), 1u);
          atomicAdd(a.acc.emq + gc * MAXV + (iq - 1), 1u);
          atomicAdd(a.acc.emph + gc * MAXV + (iph - 1), 1u);
        }
      }
    }
    double VR[3], A1[3], A2[3], A4[3], x2[3], x4[3];
    for (int k = 0; k < 3; ++k) VR[k] = vpar * ep[k] + vps * epp[k] + vphs * eph[k];
    ena_acc(a, x, A1);
    for (int k = 0; k < 3; ++k) x2[k] = x[k] + hh * VR[k];
    ena_acc(a, x2, A2);
    for (int k = 0; k < 3; ++k) x4[k] = x[k] + h * VR[k] + hsq2 * A1[k];
    ena_acc(a, x4, A4);
    double VN[3], xN[3];
    for (int k = 0; k < 3; ++k) {
      VN[k] = VR[k] + h6 * (A1[k] + 2.0 * A2[k] + 2.0 * A2[k] + A4[k]);
      const double vk2 = VR[k] + hh * A1[k], vk4 = VR[k] + h * A2[k];
      xN[k] = x[k] + h6 * (VR[k] + 2.0 * vk2 + 2.0 * vk2 + vk4);
    }
    ena_geo(xN, ct, st, cp, sp, q, ir);
    dipole_frame(ct, st, cp, sp, ep, epp, eph);
    const double vparN = ep[0] * VN[0] + ep[1] * VN[1] + ep[2] * VN[2];
    const double vpN = fabs(epp[0] * VN[0] + epp[1] * VN[1] + epp[2] * VN[2]);
    const double vphN = eph[0] * VN[0] + eph[1] * VN[1];
    a.ena.x[e] = xN[0];
    a.ena.y[e] = xN[1];
    a.ena.z[e] = xN[2];
    a.ena.vx[e] = vparN * ep[0] + vpN * epp[0] + vphN * eph[0];
    a.ena.vy[e] = vparN * ep[1] + vpN * epp[1] + vphN * eph[1];
    a.ena.vz[e] = vparN * ep[2] + vpN * epp[2] + vphN * eph[2];
    a.ena.vps[e] = vps;
    a.ena.vphs[e] = vphs;
    a.ena.qind[e] = qi;
  }
  }  // units
}

// ENA moments of one master step from the ENA counts and (Vp, Vq, Vphi)
// marginals (ZerothENAMoment .. SecondPHIENAMoment _8_10_1 .. _8_10_8 with
// NonUniform3DIntegratorSub _8_9): integrands hVp hVq hVphi F (.) at the
// bin centres, M1 = MM/M0, M2 = 6.242e18 (ms/2) MM/M0 centred on M1.  One
// warp per cell.
__global__ void __launch_bounds__(256) k_ena_moments(const TubeD *tubes,
                                                     const int *cell_tube,
                                                     CellTables c, Accum acc) {
  const int64_t g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t NC = c.ncell_total;
  if (g >= NC) return;  // whole warp
  const TubeD &T = tubes[cell_tube[g]];
  const double ms = T.ms;
  const double w = T.nsnormfac / c.d3xC[g];
  const double NqENA = (double)acc.ecnt[g] * w;
  const unsigned *mp = acc.emp + g * MAXV, *mq = acc.emq + g * MAXV,
                 *mph = acc.emph + g * MAXV;
  const int np = c_evg.n1, nq = c_evg.npar, nph = c_evg.n2;
  auto centre = [](const double *e, int k) { return 0.5 * (e[k] + e[k + 1]); };
  double N = 0.0, Sp = 0.0, Sq = 0.0, Sph = 0.0;
  for (int k = lane; k < np; k += 32) {
    N += (double)mp[k];
    Sp += w * centre(c_evg.e1, k) * (double)mp[k];
  }
  for (int k = lane; k < nq; k += 32) Sq += w * centre(c_evg.epar, k) * (double)mq[k];
  for (int k = lane; k < nph; k += 32) Sph += w * centre(c_evg.e2, k) * (double)mph[k];
  N = warp_sum(N);
  Sp = warp_sum(Sp);
  Sq = warp_sum(Sq);
  Sph = warp_sum(Sph);
  const double M0 = (NqENA == 0.0) ? 0.0 : w * N;
  double m1p = 0.0, m1q = 0.0, m1ph = 0.0, tp = 0.0, tq = 0.0, tph = 0.0;
  if (M0 != 0.0) {
    m1p = Sp / M0;
    m1q = Sq / M0;
    m1ph = Sph / M0;
    for (int k = lane; k < np; k += 32) {
      const double d = m1p - centre(c_evg.e1, k);
      tp += w * fabs(d * d) * (double)mp[k];
    }
    for (int k = lane; k < nq; k += 32) {
      const double d = m1q - centre(c_evg.epar, k);
      tq += w * fabs(d * d) * (double)mq[k];
    }
    for (int k = lane; k < nph; k += 32) {
      const double d = m1ph - centre(c_evg.e2, k);
      tph += w * fabs(d * d) * (double)mph[k];
    }
    tp = warp_sum(tp);
    tq = warp_sum(tq);
    tph = warp_sum(tph);
  }
  if (lane == 0) {
    const double eV = 6.242e18, f = M0 != 0.0 ? eV * (ms / 2.0) / M0 : 0.0;
    double *mom = c.mom;
    mom[KAOS_ENA_NQ * NC + g] = NqENA;
    mom[KAOS_ENA_M0 * NC + g] = M0;
    mom[KAOS_ENA_M1P * NC + g] = m1p;
    mom[KAOS_ENA_M1Q * NC + g] = m1q;
    mom[KAOS_ENA_M1PHI * NC + g] = m1ph;
    mom[KAOS_ENA_M2 * NC + g] = (tp + tq + tph) * f;
    mom[KAOS_ENA_M2P * NC + g] = tp * f;
    mom[KAOS_ENA_M2Q * NC + g] = tq * f;
    mom[KAOS_ENA_M2PHI * NC + g] = tph * f;
  }
}

}  // namespace kaos
