// kaos_api.cu -- host side of the C-ABI (include/kaos_gpu.h): device memory
// for the particles and per-cell tables, and the per-step launch sequence
// that replaces the body of KineticSolverSub (_8_KineticSolver.f90:54-239).
//
// Everything stays resident in HBM across calls; the host only issues
// launches on the handle's stream and reads results on request.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "kaos_cx.cuh"
#include "kaos_tube.cuh"

using namespace kaos;

namespace {

constexpr int PUSH_THREADS = 256;
constexpr int PUSH_ITEMS = 8;
constexpr int BC_THREADS = 256;
// Removal at a master step marks the escaped ions DEAD in place; the ion
// arrays are compacted (order-preserving) every BC_COMPACT_EVERY master
// steps, or earlier when an injection could overflow a tube's capacity.
constexpr int BC_COMPACT_EVERY = 8;
// cells per tube: the per-cell tables of a tube live in shared memory (the
// mixed push holds 92 bytes per cell, the collision-count kernel 64)
constexpr int MAX_CELLS = 2048;
// push work-item sizes the autotuner tries (ions per item); an item's ions
// lie in one charge-exchange selection chunk
constexpr int NCHUNKS = 3;
constexpr int CHUNKS[NCHUNKS] = {1024, 2048, 4096};
static_assert(CX_CHUNK % 4096 == 0 && CX_CHUNK % (PUSH_THREADS * PUSH_ITEMS) == 0,
              "chunk sizes");
// k_push_ena's shared memory: the tube's cell edges, the per-tube unit prefix
static size_t ena_push_smem(int nq, int ntubes) {
  return (size_t)(nq + 1) * sizeof(double) + (size_t)(ntubes + 1) * sizeof(int);
}
// k_cx_convert's shared memory: conversions still owed per cell, per-warp
// per-cell counts (8 warps), the chunk's Qindk1
static size_t cx_convert_smem(int nq) {
  return ((size_t)9 * nq + CX_CHUNK) * sizeof(unsigned);
}

// Positive root u = r/RE of q^2 u^4 + u/p - 1 = 0: closed form of the
// depressed resolvent cubic in hyperbolic form, then Newton polish.
double host_quartic_u(double q, double p) {
  if (q == 0.0) return p;
  double Cp = 1.0 / (p * q * q);
  double eps = 4.0 / (3.0 * q * q);
  double t = (Cp * Cp / 2.0) / (eps * std::sqrt(eps));
  double sigma = 2.0 * std::sqrt(eps) * std::sinh(std::asinh(t) / 3.0);
  double mu = std::sqrt(sigma);
  double u = (-mu + std::sqrt(-sigma + 2.0 * Cp / mu)) / 2.0;
  for (int k = 0; k < 4; ++k) {
    double f = q * q * u * u * u * u + u / p - 1.0;
    double fp = 4.0 * q * q * u * u * u + 1.0 / p;
    u -= f / fp;
  }
  return u;
}

void host_rho_z(double q, double p, double *rho, double *z) {
  double u = host_quartic_u(q, p);
  double st = std::sqrt(u / p), ct = q * u * u, r = u * RE;
  *rho = r * st;
  *z = r * ct;
  if (std::fabs(*rho) < 1e-6) *rho = 0.0;
  if (std::fabs(*z) < 1e-6) *z = 0.0;
}

template <typename T>
struct DBuf {
  T *p = nullptr;
  size_t n = 0;
};

}  // namespace

struct kaos_handle {
  kaos_params_c P{};
  int ntubes = 0;
  int mixed = 0;
  int kick64 = 0;  // mixed push with the FP64 heating kick
  int three_d = 1;
  int nv = 0;
  int64_t ncell = 0;
  std::vector<TubeD> th;          // host copy of tube descriptors
  std::vector<std::vector<double>> host_cells;  // for getters
  VGridC vg{};
  VGridC evg{};  // ENA velocity grid (Vp = 1, Vq = par, Vphi = 2)
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  // side stream of the ENA push, which runs beside the ion push (fork after
  // the charge exchange, join before anything that follows the pushes)
  cudaStream_t s2 = nullptr;
  cudaEvent_t efork = nullptr, ejoin = nullptr;
  // device
  TubeD *d_tubes = nullptr;
  int *d_blk_tube = nullptr;
  int64_t *d_blk_start = nullptr;
  int *d_tube_blk0 = nullptr;
  int nblk = 0;
  std::vector<int> tube_blk0;
  int64_t *d_nlive = nullptr, *d_nlive_new = nullptr;
  uint64_t *d_next_id = nullptr;
  int64_t *d_blkcnt = nullptr, *d_blkoff = nullptr;
  unsigned long long *d_lb_out = nullptr, *d_ub_out = nullptr,
                     *d_lb_in = nullptr, *d_ub_in = nullptr;
  uint32_t *d_status = nullptr;
  std::vector<void *> allocs;
  CellTables ct{};
  Accum acc{};
  Ions ion[2]{};
  int cur = 0;
  // ENA population (charge exchange)
  Enas ena[2]{};
  int ecur = 0;
  int64_t *d_nena = nullptr, *d_nena_new = nullptr;
  int *d_eblk_tube = nullptr, *d_tube_eblk0 = nullptr;
  int64_t *d_eblk_start = nullptr, *d_eblkcnt = nullptr, *d_eblkoff = nullptr;
  int neblk = 0;
  unsigned long long *d_lbe_out = nullptr, *d_ube_out = nullptr;
  int *d_cx_tube = nullptr, *d_tube_cx0 = nullptr;
  unsigned *d_cxconv = nullptr;
  int64_t *d_cxbase = nullptr;
  int64_t *d_cx_start = nullptr;
  unsigned *d_cxc = nullptr, *d_cxo = nullptr;
  int *d_cxend = nullptr;
  int *d_tube_done = nullptr;  // per tube: charge-exchange cell scans done
  int *d_cx_list = nullptr, *d_cx_nlist = nullptr, *d_tube_active = nullptr;
  int *d_cx_chunks = nullptr;       // chunks with conversions this step
  unsigned *d_cx_nchunk = nullptr;  // their count, blocks that read it
  int cx_blocks = 0;                // k_cx_convert: one resident wave
  // convection: device staging of the moves of one master step (allocated
  // at the first move) and its host side
  double *d_conv_stage = nullptr, *d_conv_pnew = nullptr;
  TubeD *d_conv_td = nullptr;
  int *d_conv_tube = nullptr;
  struct ConvHost {
    double *stage = nullptr;  // pinned: [move][table][nqmax]
    std::vector<double> pnew;
    std::vector<TubeD> td;
    std::vector<int> tube;
  } conv_host;
  int *d_cell_tube = nullptr, *d_cell_q = nullptr;  // global cell -> (tube, cell)
  int ncx = 0;
  int64_t n = 0;      // computational steps taken
  int export_on = 0;
  int have_import = 0;
  int loaded = 0;
  int graph = 0;
  // CUDA graphs of whole steps: kernels replayed from a graph read the step
  // number from d_step (advanced by the first kernel of every step)
  uint32_t *d_step = nullptr;
  int capturing = 0;
  int dstep_valid = 0;
  // charge exchange idle for the current master interval: the last master
  // step listed no converting cell and left no ENA.  Its ordinary steps
  // then launch no selection, conversion or ENA push, the pushes count no
  // Qindk1 for the selection and store no Qindk1 or k4 point for it (master
  // steps keep all of it: their moments decide the next interval).  Decided
  // on the host from cx_stat, copied back after every master step.
  int cx_idle = 0;
  int cx_stat_pending = 0;
  int64_t *cx_stat = nullptr;  // pinned: [0] listed cells, [1..ntubes] ENAs
  struct StepGraph {
    cudaGraphExec_t exec = nullptr;
    int64_t launches = 0;
  };
  std::map<uint64_t, StepGraph> graphs;
  // all binning accumulators in one block; optional cross-rank reduction
  unsigned *acc_base = nullptr;
  int64_t acc_len = 0;
  kaos_reduce_fn reduce_fn = nullptr;
  void *reduce_ctx = nullptr;
  int rank = 0, nranks = 1;          // share of the charge-exchange counts
  std::vector<uint64_t> id_base;     // first ion id per tube
  // tube moves (kaos_update_tube) applied at the next master step
  struct PendingTube {
    int tube;
    TubeD d;
    std::vector<std::vector<double>> tables;  // in CONV_TABLES order
  };
  std::vector<PendingTube> pending, applied;
  // push work items: (tube, chunk of ions) maps, one per candidate chunk
  struct WorkMap {
    int chunk = 0, n = 0;
    int *d_tube = nullptr;
    int64_t *d_start = nullptr;
  };
  WorkMap wmap[NCHUNKS];
  int wsel = 1;          // chosen map (CHUNKS[wsel] ions per item)
  int persistent = 0;    // persistent grid striding over the items
  int tune_pending = 1;  // autotune before the next step
  int regsel = 0;        // mixed push register budget: 0 = 64, 1 = 80, 2 = 72
  int regsel_master = 0; // the same for the master-step variant of the push
  int nsm = 0;
  // resident push blocks per SM per (master-step variant, budget); 0: unknown
  int occ[2][3] = {{0, 0, 0}, {0, 0, 0}};
  int64_t ion_len = 0;   // length of every ion array (all tubes' capacity)
  double last_ms = 0.0;
  int64_t launches = 0;
  std::vector<cudaEvent_t> pev;  // event pairs around push launches
  int npev = 0;
  double push_ms = 0.0;
  // deferred compaction: master steps since the last one, the decision of
  // master step bc_for, and per tube an upper bound of the occupied slots
  int bc_since = 0;
  int64_t bc_for = -1;
  int bc_compact = 1;
  std::vector<int64_t> bc_bound;
  char err[512] = {0};
};

namespace {

// The handle whose velocity grids were copied last into c_vg / c_evg; a
// step of another handle, or after a grid change, copies its own.
std::atomic<const kaos_handle *> g_grid_owner{nullptr};

int fail(kaos_handle *h, int code, const char *fmt, ...) {
  if (h) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(h->err, sizeof(h->err), fmt, ap);
    va_end(ap);
  }
  return code;
}

#define CK(call)                                                              \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess)                                                    \
      return fail(h, KAOS_ERR_CUDA, "%s: %s (%s:%d)", #call,                 \
                  cudaGetErrorString(e_), __FILE__, __LINE__);                \
  } while (0)

template <typename T>
int dalloc(kaos_handle *h, T **p, size_t n) {
  void *q = nullptr;
  size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e != cudaSuccess)
    return fail(h, KAOS_ERR_CUDA, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  cudaMemset(q, 0, bytes);
  h->allocs.push_back(q);
  *p = (T *)q;
  return KAOS_OK;
}

int upload(kaos_handle *h, double **dst, const std::vector<double> &v) {
  int rc = dalloc(h, dst, v.size());
  if (rc) return rc;
  CK(cudaMemcpy(*dst, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice));
  return KAOS_OK;
}

bool is_master(const kaos_handle *h, int64_t n) {
  return n >= 2 && (n % h->P.ndatfac) == 0;
}

int max_nq(const kaos_handle *h) {
  int m = 0;
  for (auto &t : h->th) m = std::max(m, t.nq);
  return m;
}

PushArgs push_args(kaos_handle *h) {
  PushArgs a{};
  a.tubes = h->d_tubes;
  const kaos_handle::WorkMap &M = h->wmap[h->wsel];
  a.blk_tube = M.d_tube;
  a.blk_start = M.d_start;
  a.nitems = M.n;
  a.chunk = M.chunk;
  a.nqs = max_nq(h);
  a.nlive = h->d_nlive;
  a.ion = h->ion[h->cur];
  a.ct = h->ct;
  a.acc = h->acc;
  a.h = h->P.h;
  a.ms = h->P.ms;
  a.qs = h->P.qs;
  a.seed = h->P.seed;
  a.ff.mirror = h->P.MIRRORflag == 1;
  a.ff.grav = h->P.GRAVflag == 1;
  a.ff.eamb = h->P.EAMBflag == 1;
  a.ff.eambsign = h->P.EAMBSIGNflag == 1;
  a.icr = h->P.ICRflag == 1;
  a.icrcoh = h->P.ICRCOHERENCEflag == 1;
  a.status = h->d_status;
  a.exporting = h->export_on;
  a.cxc = nullptr;  // set by the pushes whose Qindk1 feeds a selection
  a.tube_cx0 = h->d_tube_cx0;
  a.cx_stride = max_nq(h);
  a.cx_chunk = CX_CHUNK;
  a.dstep = h->capturing ? h->d_step : nullptr;
  for (int r = 0; r < 10; ++r) {  // Philox key schedule of the seed
    a.rk[2 * r] = (uint32_t)h->P.seed + (uint32_t)r * KAOS_PHILOX_W0;
    a.rk[2 * r + 1] = (uint32_t)(h->P.seed >> 32) + (uint32_t)r * KAOS_PHILOX_W1;
  }
  return a;
}

TubeArgs tube_args(kaos_handle *h, uint32_t nn) {
  TubeArgs a{};
  a.tubes = h->d_tubes;
  a.ntubes = h->ntubes;
  a.ct = h->ct;
  a.acc = h->acc;
  a.nlive = h->d_nlive;
  a.ms = h->P.ms;
  a.qs = h->P.qs;
  a.h = h->P.h;
  a.mNeut = h->P.mNeut;
  a.TNeut = h->P.TNeut;
  a.dNTe = h->P.dNTe;
  a.dNTeEND = h->P.dNTeEND;
  a.seed = h->P.seed;
  a.nn = nn;
  a.dstep = h->capturing ? h->d_step : nullptr;
  a.ndatfac = h->P.ndatfac;
  a.three_d = h->three_d;
  a.eamb = h->P.EAMBflag == 1;
  a.grav = h->P.GRAVflag == 1;
  a.eapressure = h->P.EAPRESSUREflag == 1;
  a.eambsign = h->P.EAMBSIGNflag == 1;
  a.eambself = h->P.EAMBSELFCONSISTflag == 1;
  a.momfilter = h->P.MOMENTFILTERflag == 1;
  a.qexchange = h->P.QEXCHANGEflag == 1;
  a.cenpar = h->P.PHASEENERGYPARIONMOMENTCENTERflag == 1;
  a.cenperp = h->P.PHASEENERGYPERPIONMOMENTCENTERflag == 1;
  a.fpM0 = h->P.M0MAfilterPt;
  a.fpM1par = h->P.M1ParMAfilterPt;
  a.fpM1p1 = h->P.M1Perp1MAfilterPt;
  a.fpM1p2 = h->P.M1Perp2MAfilterPt;
  a.fpM2par = h->P.M2ParMAfilterPt;
  return a;
}

int launch_push(kaos_handle *h, const PushArgs &a) {
  const int nq = max_nq(h);
  const bool timed = !h->capturing;  // no per-push events inside a graph
  if (timed && (int)h->pev.size() < 2 * (h->npev + 1)) {
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    h->pev.push_back(e0);
    h->pev.push_back(e1);
  }
  if (timed) CK(cudaEventRecord(h->pev[2 * h->npev], h->s));
  size_t smem = (size_t)(2 * nq + 1) * sizeof(double) + (size_t)nq * sizeof(unsigned);
  if (h->mixed)  // + one double of padding before the 16-byte aligned floats
    smem += (size_t)(6 * nq + 1) * sizeof(double) + (size_t)10 * nq * sizeof(float);
  smem += (size_t)BIN_WIN * (1 + h->vg.npar + h->vg.n1 + (h->three_d ? h->vg.n2 : 0)) *
          sizeof(unsigned);  // block-private binning window
  const bool bins_variant = a.bin || a.prologue || a.bin_only || !h->three_d;
  if (h->mixed && bins_variant) smem += BINS_SMEM_BYTES;  // FP64 edges + tables
  const int ms = (a.bin || a.prologue || a.bin_only) ? 1 : 0;
  const int rs = h->mixed ? (ms ? h->regsel_master : h->regsel) : 0, ps = h->persistent;
  // kernel variant: [master-step work][three_d][register budget][persistent];
  // the budgets: 64 registers (4 blocks of 256 threads per SM), 80 (3
  // blocks of 256), 72 (7 blocks of 128)
  using KFn = void (*)(PushArgs);
#define KAOS_K32(M, D, K)                                                     \
  {{k_push32<D, 256, 4, false, M, K>, k_push32<D, 256, 4, true, M, K>},      \
   {k_push32<D, 256, 3, false, M, K>, k_push32<D, 256, 3, true, M, K>},      \
   {k_push32<D, 128, 7, false, M, K>, k_push32<D, 128, 7, true, M, K>}}
  // [FP64 heating kick][master-step work][three_d][register budget][persistent]
  static const KFn k32[2][2][2][3][2] = {
      {{KAOS_K32(false, false, false), KAOS_K32(false, true, false)},
       {KAOS_K32(true, false, false), KAOS_K32(true, true, false)}},
      {{KAOS_K32(false, false, true), KAOS_K32(false, true, true)},
       {KAOS_K32(true, false, true), KAOS_K32(true, true, true)}}};
#undef KAOS_K32
  const int nt = rs == 2 ? 128 : PUSH_THREADS;
  static const KFn k64[2][2] = {{k_push64<false, false>, k_push64<false, true>},
                                {k_push64<true, false>, k_push64<true, true>}};
  const KFn fn = h->mixed ? k32[h->kick64][ms][h->three_d][rs][ps] : k64[h->three_d][ps];
  if (smem > 48 * 1024)
    CK(cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int &occ = h->occ[h->mixed ? ms : 0][rs];
  if (!occ) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void *)fn, nt, smem));
    occ = std::max(occ, 1);
  }
  const int grid = ps ? std::min(a.nitems, h->nsm * occ) : a.nitems;
  if (grid > 0) fn<<<grid, nt, smem, h->s>>>(a);
  if (timed) {
    CK(cudaEventRecord(h->pev[2 * h->npev + 1], h->s));
    h->npev++;
  }
  h->launches++;
  CK(cudaGetLastError());
  return KAOS_OK;
}

int zero_accum(kaos_handle *h) {
  const int64_t nc = h->ncell;
  CK(cudaMemsetAsync(h->acc_base, 0, (size_t)h->acc_len * sizeof(unsigned), h->s));
  if (h->export_on && h->acc.hist)
    CK(cudaMemsetAsync(h->acc.hist, 0, nc * (int64_t)h->nv * sizeof(unsigned), h->s));
  return KAOS_OK;
}

// The per-cell tables of one tube, in the order of CellTables' pointers
// listed by conv_table_ptr (the same values kaos_create builds).
constexpr int CONV_TABLES = 28;
std::vector<std::vector<double>> tube_tables(const kaos_tube_c &T, const TubeD &d,
                                             const kaos_params_c &p) {
  std::vector<std::vector<double>> v(CONV_TABLES);
  auto app = [&](int k, const double *src, double dflt) {
    for (int c = 0; c < T.nq; ++c) v[k].push_back(src ? src[c] : dflt);
  };
  app(0, T.qGL, 0); app(1, T.qGH, 0); app(2, T.qGC, 0); app(3, T.hqC, 0);
  app(4, T.dqC, 0); app(5, T.d3xC, 1); app(6, T.rGC, 0); app(7, T.thetaGC, 0);
  app(8, T.ellGC, 1); app(9, T.TeG, 0); app(10, T.TsG, 0); app(11, T.nsnormCNeut, 0);
  app(12, T.lambdaPerp, 0); app(13, T.EtaLH, 0); app(14, T.XiPerp1, 0);
  app(15, T.XiPerp2, 0); app(16, T.S0, 0); app(17, T.OmegaG0, 1);
  app(18, T.ChiPerp1, 0); app(19, T.ChiPerp2, 0);
  for (int c = 0; c < T.nq; ++c) {
    v[20].push_back(host_quartic_u(T.qGL[c], T.pG));
    v[21].push_back(host_quartic_u(T.qGH[c], T.pG));
    const double pre = (d.qs * d.qs / (2.0 * d.ms * d.ms)) *
                       (T.S0 ? T.S0[c] : 0.0) * (T.EtaLH ? T.EtaLH[c] : 0.0);
    v[22].push_back(p.h * std::sqrt(pre * (T.XiPerp1 ? T.XiPerp1[c] : 0.0) / PI));
    v[23].push_back(p.h * std::sqrt(pre * (T.XiPerp2 ? T.XiPerp2[c] : 0.0) / PI));
    v[24].push_back(0.5 * (T.ChiPerp1 ? T.ChiPerp1[c] : 0.0));
    v[25].push_back(0.5 * (T.ChiPerp2 ? T.ChiPerp2[c] : 0.0));
    v[26].push_back(T.OmegaG0 && T.OmegaG0[c] != 0.0 ? 1.0 / T.OmegaG0[c] : 0.0);
    v[27].push_back(host_quartic_u(0.5 * (T.qGL[c] + T.qGH[c]), T.pG));
  }
  return v;
}

const double *conv_table_ptr(const CellTables &c, int k) {
  const double *p[CONV_TABLES] = {c.qGL, c.qGH, c.qGC, c.hqC, c.dqC, c.d3xC, c.rGC,
                                  c.thetaGC, c.ellGC, c.TeG, c.TsG, c.nsnormCNeut,
                                  c.lambdaPerp, c.EtaLH, c.XiPerp1, c.XiPerp2, c.S0,
                                  c.OmegaG0, c.ChiPerp1, c.ChiPerp2, c.uL, c.uH,
                                  c.hK1, c.hK2, c.hc1, c.hc2, c.hiom0, c.uM};
  return p[k];
}

// Move the tubes given to kaos_update_tube, all in two launches: re-project
// their ions with the old tables and descriptors (k_convect_many), then put
// the new tables and descriptors in place (k_apply_tables) from one staging
// copy.
static int sm_count(kaos_handle *h);

int apply_pending_tubes(kaos_handle *h) {
  static_assert(CONV_TABLES == CONV_NTAB, "table count");
  const int np = (int)h->pending.size();
  if (!np) return KAOS_OK;
  const int nqm = max_nq(h);
  int rc;
  const size_t stage_len = (size_t)h->ntubes * CONV_TABLES * nqm;
  if (!h->d_conv_stage) {  // staging for every entry moving at once
    if ((rc = dalloc(h, &h->d_conv_stage, stage_len)) ||
        (rc = dalloc(h, &h->d_conv_td, (size_t)h->ntubes)) ||
        (rc = dalloc(h, &h->d_conv_tube, (size_t)h->ntubes)) ||
        (rc = dalloc(h, &h->d_conv_pnew, (size_t)h->ntubes)))
      return rc;
    CK(cudaMallocHost((void **)&h->conv_host.stage, stage_len * sizeof(double)));
  }
  // the moves, their new descriptors and tables in host staging (the tables
  // in pinned memory, copied asynchronously; the staging is next written at
  // the next move, after the step that applied this one has finished)
  auto &S = h->conv_host;
  S.td.resize(np);
  S.tube.resize(np);
  S.pnew.resize(np);
  for (int p = 0; p < np; ++p) {
    const auto &pt = h->pending[p];
    S.td[p] = pt.d;
    S.tube[p] = pt.tube;
    S.pnew[p] = pt.d.pG;
    for (int k = 0; k < CONV_TABLES; ++k)
      std::copy(pt.tables[k].begin(), pt.tables[k].end(),
                S.stage + ((size_t)p * CONV_TABLES + k) * nqm);
  }
  CK(cudaMemcpyAsync(h->d_conv_stage, S.stage, (size_t)np * CONV_TABLES * nqm * sizeof(double),
                     cudaMemcpyHostToDevice, h->s));
  CK(cudaMemcpyAsync(h->d_conv_td, S.td.data(), np * sizeof(TubeD), cudaMemcpyHostToDevice, h->s));
  CK(cudaMemcpyAsync(h->d_conv_tube, S.tube.data(), np * sizeof(int), cudaMemcpyHostToDevice, h->s));
  CK(cudaMemcpyAsync(h->d_conv_pnew, S.pnew.data(), np * sizeof(double), cudaMemcpyHostToDevice, h->s));
  // re-project the ions with the old tables and descriptors, then swap them
  ConvManyArgs ca{};
  ca.tubes = h->d_tubes;
  ca.tube = h->d_conv_tube;
  ca.p_new = h->d_conv_pnew;
  ca.nlive = h->d_nlive;
  ca.ion = h->ion[h->cur];
  ca.ct = h->ct;
  ca.mixed = h->mixed;
  k_convect_many<<<dim3(std::max(1, sm_count(h) * 16 / np), np), 256, 0, h->s>>>(ca);
  TableApplyArgs ta{};
  for (int k = 0; k < CONV_TABLES; ++k) ta.dst[k] = (double *)conv_table_ptr(h->ct, k);
  ta.stage = h->d_conv_stage;
  ta.td = h->d_conv_td;
  ta.tube = h->d_conv_tube;
  ta.tubes = h->d_tubes;
  ta.nqmax = nqm;
  k_apply_tables<<<dim3(CONV_TABLES, np), 256, 0, h->s>>>(ta);
  h->launches += 2;
  CK(cudaGetLastError());
  for (const auto &pt : h->pending) h->th[pt.tube] = pt.d;
  return KAOS_OK;
}

// A tube split across ranks: the caller's hook sums the binning
// accumulators of all ranks in place before the moments are taken.
int reduce_accum(kaos_handle *h) {
  if (!h->reduce_fn) return KAOS_OK;
  CK(cudaStreamSynchronize(h->s));
  const int rc = h->reduce_fn(h->reduce_ctx, h->acc_base, h->acc_len, (void *)h->s);
  if (rc) return fail(h, KAOS_ERR_CUDA, "accumulator reduction hook returned %d", rc);
  return KAOS_OK;
}

CxArgs cx_args(kaos_handle *h);

int launch_moments(kaos_handle *h, uint32_t nn) {
  TubeArgs ta = tube_args(h, nn);
  const int cells_per_block = 256 / 32;
  k_cell_moments<<<(int)((h->ncell + cells_per_block - 1) / cells_per_block), 256, 0, h->s>>>(
      ta, h->d_cell_tube);
  h->launches++;
  if (ta.qexchange) {
    size_t smem = (size_t)8 * max_nq(h) * sizeof(double);
    k_collision_counts<<<h->ntubes, 256, smem, h->s>>>(ta);
    // the cells that will convert ions until the next master step
    CK(cudaMemsetAsync(h->d_cx_nlist, 0, sizeof(int), h->s));
    CK(cudaMemsetAsync(h->d_tube_active, 0, h->ntubes * sizeof(int), h->s));
    k_cx_list<<<(int)((h->ncell + 255) / 256), 256, 0, h->s>>>(cx_args(h), h->d_cell_tube,
                                                             h->ncell);
    h->launches += 2;
    // the next interval's activity (read on the host before its first step)
    CK(cudaMemcpyAsync(h->cx_stat, h->d_cx_nlist, sizeof(int), cudaMemcpyDeviceToHost, h->s));
    CK(cudaMemcpyAsync(h->cx_stat + 1, h->d_nena, h->ntubes * sizeof(int64_t),
                       cudaMemcpyDeviceToHost, h->s));
    h->cx_stat_pending = 1;
    if (nn > 1) {  // ENA statistics from the second master step on
      k_ena_moments<<<(int)((h->ncell + cells_per_block - 1) / cells_per_block), 256, 0, h->s>>>(
          h->d_tubes, h->d_cell_tube, h->ct, h->acc);
      h->launches++;
    }
  }
  CK(cudaGetLastError());
  return KAOS_OK;
}

int launch_fields(kaos_handle *h, int te_update) {
  TubeArgs ta = tube_args(h, 0);
  ta.te_update = te_update;
  ta.have_import = 0;
  size_t smem = (size_t)3 * max_nq(h) * sizeof(double);
  k_fields<<<h->ntubes, 256, smem, h->s>>>(ta);
  h->launches++;
  CK(cudaGetLastError());
  return KAOS_OK;
}

Fields ion_fields(kaos_handle *h, int from, int to) {
  Fields F{};
  const Ions &A = h->ion[from], &B = h->ion[to];
  auto add = [&](void *s, void *d, int sz) {
    if (s) F.f[F.n++] = Field{s, d, sz};
  };
  if (h->mixed) {
    add(A.x, B.x, 8); add(A.vpar, B.vpar, 8); add(A.v12, B.v12, 16);
    add(A.ffl, B.ffl, 8); add(A.fqk4, B.fqk4, 4);
  } else {
    add(A.rho, B.rho, 8); add(A.z, B.z, 8); add(A.vpar, B.vpar, 8);
    add(A.v1, B.v1, 8); add(A.v2, B.v2, 8); add(A.aea, B.aea, 8);
    add(A.ag, B.ag, 8); add(A.qk4, B.qk4, 8);
    add(A.rho4, B.rho4, 8); add(A.z4, B.z4, 8);
  }
  add(A.qind, B.qind, 4);
  add(A.vb, B.vb, 4);
  add(A.id, B.id, 8);
  return F;
}

// Staging for the host transfers of kaos_load_particles and
// kaos_get_particles: four 8-byte-per-slot arrays and the Qindk1 array of
// the spare buffer set at tube t's segment (the spare set holds nothing
// between steps; the packing and the autotuner use it only inside a step).
void spare_slots(kaos_handle *h, int t, double *d[4], int32_t **qi) {
  Ions &S = h->ion[1 - h->cur];
  const int64_t o = h->th[t].off;
  if (h->mixed) {
    d[0] = S.x + o;
    d[1] = S.vpar + o;
    d[2] = (double *)(S.ffl + o);
  } else {
    d[0] = S.rho + o;
    d[1] = S.z + o;
    d[2] = S.vpar + o;
  }
  d[3] = (double *)(S.id + o);
  if (qi) *qi = S.qind + o;
}

// Ions one master step's injection may add to tube t.
int64_t inject_max(const kaos_handle *h, int t) {
  const TubeD &T = h->th[t];
  int64_t k = 0;
  if (h->P.LBCONDITIONflag == 1) k += std::max<int64_t>(0, std::llround(T.nsnormCLB));
  if (h->P.UBCONDITIONflag == 1) k += std::max<int64_t>(0, std::llround(T.nsnormCUB));
  return k;
}

// Whether master step n compacts the ion arrays (decided once per step, before
// any capture of it): every BC_COMPACT_EVERY master steps, or when the next
// injection could exceed a tube's capacity after the occupied slots are read
// back (outside a capture only; inside one the step compacts).
int bc_decide(kaos_handle *h, int64_t n) {
  if (h->bc_for == n) return h->bc_compact;
  int c = h->bc_since + 1 >= BC_COMPACT_EVERY;
  bool tight = false;
  for (int t = 0; t < h->ntubes && !c; ++t)
    tight = tight || h->bc_bound[t] + inject_max(h, t) > h->th[t].cap;
  if (!c && tight) {
    std::vector<int64_t> nl(h->ntubes);
    if (h->capturing || cudaStreamSynchronize(h->s) != cudaSuccess ||
        cudaMemcpy(nl.data(), h->d_nlive, h->ntubes * sizeof(int64_t),
                   cudaMemcpyDeviceToHost) != cudaSuccess) {
      c = 1;
    } else {
      for (int t = 0; t < h->ntubes; ++t) {
        h->bc_bound[t] = nl[t];
        c = c || nl[t] + inject_max(h, t) > h->th[t].cap;
      }
    }
  }
  h->bc_for = n;
  h->bc_compact = c;
  return c;
}

// Host bookkeeping of a master step's removal and injection (eager, capture
// and replay alike).
void bc_after(kaos_handle *h, int compact) {
  if (compact) {
    h->cur = 1 - h->cur;
    h->bc_since = 0;
  } else {
    ++h->bc_since;
  }
  for (int t = 0; t < h->ntubes; ++t) h->bc_bound[t] += inject_max(h, t);
}

int launch_boundary(kaos_handle *h, int compact) {
  if (!compact) {
    BcArgs b{};
    b.tubes = h->d_tubes;
    b.blk_tube = h->d_blk_tube;
    b.blk_start = h->d_blk_start;
    b.chunk = PUSH_THREADS * PUSH_ITEMS;
    b.nlive = h->d_nlive;
    b.lb_out = h->d_lb_out;
    b.ub_out = h->d_ub_out;
    b.qind_w = h->ion[h->cur].qind;
    b.x_w = h->mixed ? h->ion[h->cur].x : nullptr;
    CK(cudaMemsetAsync(h->d_lb_out, 0, h->ntubes * sizeof(unsigned long long), h->s));
    CK(cudaMemsetAsync(h->d_ub_out, 0, h->ntubes * sizeof(unsigned long long), h->s));
    CK(cudaMemsetAsync(h->d_lb_in, 0, h->ntubes * sizeof(unsigned long long), h->s));
    CK(cudaMemsetAsync(h->d_ub_in, 0, h->ntubes * sizeof(unsigned long long), h->s));
    k_bc_mark<<<h->nblk, BC_THREADS, 0, h->s>>>(b);
    h->launches++;
    CK(cudaGetLastError());
    return KAOS_OK;
  }
  BcArgs b{};
  b.tubes = h->d_tubes;
  b.blk_tube = h->d_blk_tube;
  b.blk_start = h->d_blk_start;
  b.tube_blk0 = h->d_tube_blk0;
  b.chunk = PUSH_THREADS * PUSH_ITEMS;
  b.nlive = h->d_nlive_new;
  b.qind = h->ion[h->cur].qind;
  b.blkcnt = h->d_blkcnt;
  b.blkoff = h->d_blkoff;
  b.lb_out = h->d_lb_out;
  b.ub_out = h->d_ub_out;
  b.fields = ion_fields(h, h->cur, 1 - h->cur);
  CK(cudaMemsetAsync(h->d_lb_out, 0, h->ntubes * sizeof(unsigned long long), h->s));
  CK(cudaMemsetAsync(h->d_ub_out, 0, h->ntubes * sizeof(unsigned long long), h->s));
  CK(cudaMemsetAsync(h->d_lb_in, 0, h->ntubes * sizeof(unsigned long long), h->s));
  CK(cudaMemsetAsync(h->d_ub_in, 0, h->ntubes * sizeof(unsigned long long), h->s));
  BcArgs bc = b;
  bc.nlive = h->d_nlive;  // count reads the live counts
  k_bc_count<<<h->nblk, BC_THREADS, 0, h->s>>>(bc);
  k_bc_scan<<<h->ntubes, 1024, 0, h->s>>>(b);    // writes nlive_new
  k_bc_scatter<<<h->nblk, BC_THREADS, 0, h->s>>>(b, h->d_nlive);
  h->launches += 3;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(h->d_nlive, h->d_nlive_new, h->ntubes * sizeof(int64_t),
                     cudaMemcpyDeviceToDevice, h->s));
  return KAOS_OK;  // the caller swaps the buffer sets (bc_after)
}

int launch_inject(kaos_handle *h, int ub) {
  InjArgs a{};
  a.tubes = h->d_tubes;
  a.ct = h->ct;
  a.acc = h->acc;
  a.ion = h->ion[h->cur];
  a.nlive = h->d_nlive;
  a.next_id = h->d_next_id;
  a.n_in = ub ? h->d_ub_in : h->d_lb_in;
  a.mixed = h->mixed;
  a.ub = ub;
  a.bin = 1;
  a.exporting = h->export_on;
  a.ms = h->P.ms;
  a.qs = h->P.qs;
  a.seed = h->P.seed;
  a.status = h->d_status;
  a.flux = h->P.FLUXINJECTIONflag == 1;
  a.stat = h->P.STATICINJECTIONflag == 1;
  if (h->P.QEXCHANGEflag == 1) {  // injected ions join the next selection
    a.cxc = h->d_cxc;
    a.tube_cx0 = h->d_tube_cx0;
    a.cx_stride = max_nq(h);
    a.cx_chunk = CX_CHUNK;
  }
  // blocks per tube: enough for the largest injection, at most 64
  int64_t kmax = 0;
  for (const TubeD &T : h->th)
    kmax = std::max(kmax, (int64_t)std::llrint(ub ? T.nsnormCUB : T.nsnormCLB));
  const int bx = (int)std::min<int64_t>(64, std::max<int64_t>(1, (kmax + 255) / 256));
  k_inject<<<dim3(bx, h->ntubes), 256, 0, h->s>>>(a);
  k_inject_commit<<<(h->ntubes + 127) / 128, 128, 0, h->s>>>(a, h->ntubes);
  h->launches += 2;
  CK(cudaGetLastError());
  return KAOS_OK;
}

CxArgs cx_args(kaos_handle *h) {
  CxArgs a{};
  a.tubes = h->d_tubes;
  a.cx_tube = h->d_cx_tube;
  a.cx_start = h->d_cx_start;
  a.tube_cx0 = h->d_tube_cx0;
  a.nlive = h->d_nlive;
  a.ct = h->ct;
  a.ion = h->ion[h->cur];
  a.ena = h->ena[h->ecur];
  a.nena = h->d_nena;
  a.cxc = h->d_cxc;
  a.cxo = h->d_cxo;
  a.cxconv = h->d_cxconv;
  a.cxbase = h->d_cxbase;
  a.cxend = h->d_cxend;
  a.tube_done = h->d_tube_done;
  a.list = h->d_cx_list;
  a.nlist = h->d_cx_nlist;
  a.chunk_list = h->d_cx_chunks;
  a.nchunk = h->d_cx_nchunk;
  a.tube_active = h->d_tube_active;
  a.rank = h->rank;
  a.nranks = h->nranks;
  a.nqmax = max_nq(h);
  a.mixed = h->mixed;
  a.ncx = h->ncx;
  a.status = h->d_status;
  return a;
}

static int sm_count(kaos_handle *h) {
  if (!h->nsm) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      h->nsm = 148;
  }
  return h->nsm;
}

// Blocks of a grid striding over n work items: a few per SM.
static int strided_grid(kaos_handle *h, int n) {
  return std::max(1, std::min(n, 4 * sm_count(h)));
}

// charge exchange at the start of a step (_8_KineticSolver.f90:95-166)
int launch_cx(kaos_handle *h) {
  CxArgs a = cx_args(h);
  const int nq = max_nq(h);
  // the per-chunk Qindk1 counts were accumulated by the previous push
  // a block per listed cell (the list length is on the device: one
  // resident wave of 256-thread blocks, striding over the list)
  k_cx_scan<<<(int)std::min<int64_t>(h->ncell, 8 * (int64_t)sm_count(h)), 256, 0, h->s>>>(
      a, h->d_cell_tube, h->d_cell_q);
  // the scan has read every count: cleared for the next push; then a block
  // per chunk with conversions
  CK(cudaMemsetAsync(h->d_cxc, 0, (size_t)h->ncx * nq * sizeof(unsigned), h->s));
  k_cx_convert<<<std::max(1, std::min(h->ncx, h->cx_blocks)), 256, cx_convert_smem(nq), h->s>>>(a);
  h->launches += 2;
  CK(cudaGetLastError());
  return KAOS_OK;
}

// The ENA push on the side stream, forked from the main stream here; the
// caller joins it (join_push_ena) after the ion push.
int launch_push_ena(kaos_handle *h, int bin) {
  CK(cudaEventRecord(h->efork, h->s));
  CK(cudaStreamWaitEvent(h->s2, h->efork, 0));
  EnaArgs a{};
  a.acc = h->acc;
  a.bin = bin;
  a.tubes = h->d_tubes;
  a.blk_tube = h->d_eblk_tube;
  a.blk_start = h->d_eblk_start;
  a.tube_blk0 = h->d_tube_eblk0;
  a.nitems = h->neblk;
  a.chunk = PUSH_THREADS * PUSH_ITEMS;
  a.sub = PUSH_ITEMS;
  a.ntubes = h->ntubes;
  a.ct_nqmax = max_nq(h);
  a.nena = h->d_nena;
  a.ct = h->ct;
  a.ena = h->ena[h->ecur];
  a.h = h->P.h;
  a.grav_GM = GG * ME;
  a.grav = h->P.GRAVflag == 1;
  k_push_ena<<<strided_grid(h, h->neblk * PUSH_ITEMS), PUSH_THREADS,
               ena_push_smem(max_nq(h), h->ntubes), h->s2>>>(a);
  h->launches++;
  CK(cudaGetLastError());
  CK(cudaEventRecord(h->ejoin, h->s2));
  return KAOS_OK;
}

int join_push_ena(kaos_handle *h) {
  CK(cudaStreamWaitEvent(h->s, h->ejoin, 0));
  return KAOS_OK;
}

int launch_boundary_ena(kaos_handle *h) {
  BcArgs b{};
  b.tubes = h->d_tubes;
  b.blk_tube = h->d_eblk_tube;
  b.blk_start = h->d_eblk_start;
  b.tube_blk0 = h->d_tube_eblk0;
  b.chunk = PUSH_THREADS * PUSH_ITEMS;
  b.nlive = h->d_nena_new;
  b.qind = h->ena[h->ecur].qind;
  b.blkcnt = h->d_eblkcnt;
  b.blkoff = h->d_eblkoff;
  b.lb_out = h->d_lbe_out;
  b.ub_out = h->d_ube_out;
  b.ena = 1;
  const Enas &A = h->ena[h->ecur], &B = h->ena[1 - h->ecur];
  Fields F{};
  F.f[F.n++] = Field{A.x, B.x, 8}; F.f[F.n++] = Field{A.y, B.y, 8};
  F.f[F.n++] = Field{A.z, B.z, 8}; F.f[F.n++] = Field{A.vx, B.vx, 8};
  F.f[F.n++] = Field{A.vy, B.vy, 8}; F.f[F.n++] = Field{A.vz, B.vz, 8};
  F.f[F.n++] = Field{A.vps, B.vps, 8}; F.f[F.n++] = Field{A.vphs, B.vphs, 8};
  F.f[F.n++] = Field{A.qind, B.qind, 4}; F.f[F.n++] = Field{A.vb, B.vb, 4};
  F.f[F.n++] = Field{A.id, B.id, 8};
  b.fields = F;
  CK(cudaMemsetAsync(h->d_lbe_out, 0, h->ntubes * sizeof(unsigned long long), h->s));
  CK(cudaMemsetAsync(h->d_ube_out, 0, h->ntubes * sizeof(unsigned long long), h->s));
  BcArgs bc = b;
  bc.nlive = h->d_nena;
  k_bc_count<<<h->neblk, BC_THREADS, 0, h->s>>>(bc);
  k_bc_scan<<<h->ntubes, 1024, 0, h->s>>>(b);
  k_bc_scatter<<<h->neblk, BC_THREADS, 0, h->s>>>(b, h->d_nena);
  h->launches += 3;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(h->d_nena, h->d_nena_new, h->ntubes * sizeof(int64_t),
                     cudaMemcpyDeviceToDevice, h->s));
  h->ecur = 1 - h->ecur;
  return KAOS_OK;
}

// kaos_sample_rng: draw i of the chosen generator, evaluated by the device
// functions the kernels call.
struct SampleArgs {
  int kind;
  uint64_t seed, id0;
  uint32_t step, c3;
  double lambda;
  int64_t n;
  double *out;
  uint32_t rk[20];  // Philox key schedule of the seed (as PushArgs.rk)
};

int sample_width(int kind) {
  return kind == KAOS_SAMPLE_PHILOX ? 4 : (kind == KAOS_SAMPLE_POISSON ? 1 : 2);
}

__global__ void k_sample_rng(SampleArgs a) {
  double *kt = kf_tables();
  if (a.kind == KAOS_SAMPLE_GAUSS64T) kf_tables_fill(kt);
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t id = a.id0 + (uint64_t)i;
    if (a.kind == KAOS_SAMPLE_PHILOX) {
      const kaos_u32x4 w = kaos_philox((uint32_t)id, (uint32_t)(id >> 32), a.step, a.c3, a.seed);
      for (int k = 0; k < 4; ++k) a.out[4 * i + k] = (double)w.v[k];
    } else if (a.kind == KAOS_SAMPLE_GAUSS32) {
      float g1, g2;
      gauss2_mix(a.rk, id, a.step, g1, g2);
      a.out[2 * i] = g1;
      a.out[2 * i + 1] = g2;
    } else if (a.kind == KAOS_SAMPLE_GAUSS64) {
      double g1, g2;
      gauss2_64(a.seed, id, a.step, KAOS_RNG_HEAT, g1, g2);
      a.out[2 * i] = g1;
      a.out[2 * i + 1] = g2;
    } else if (a.kind == KAOS_SAMPLE_GAUSS64T) {
      double g1, g2;
      gauss2_64t(a.rk, kt, id, a.step, g1, g2);
      a.out[2 * i] = g1;
      a.out[2 * i + 1] = g2;
    } else {
      a.out[i] = (double)poisson_draw(a.seed, (uint32_t)id, a.step, a.lambda);
    }
  }
}

__global__ void k_set_step(uint32_t *d, uint32_t v) { *d = v; }
__global__ void k_next_step(uint32_t *d) { *d += 1u; }

// The charge-exchange activity of the master interval that starts at the
// next step, from the list length and ENA counts the last master step
// copied back (one host wait per master interval, outside any capture).
int resolve_cx_idle(kaos_handle *h) {
  if (!h->cx_stat_pending) return KAOS_OK;
  CK(cudaStreamSynchronize(h->s));
  int64_t enas = 0;
  for (int t = 0; t < h->ntubes; ++t) enas += h->cx_stat[1 + t];
  h->cx_idle = (*(const int *)h->cx_stat == 0 && enas == 0) ? 1 : 0;
  h->cx_stat_pending = 0;
  return KAOS_OK;
}

// One computational step n = h->n + 1.
int step_once(kaos_handle *h) {
  const int64_t n = h->n + 1;
  const bool next_master = is_master(h, n + 1);
  const bool qx = h->P.QEXCHANGEflag == 1;
  int rc;
  if (h->capturing) {  // d_step: n - 1 -> n for the kernels of this step
    k_next_step<<<1, 1, 0, h->s>>>(h->d_step);
    h->launches++;
  }
  if (n == 1) {
    // KineticSolverASub: statistics of the initial state, fields, push.
    if ((rc = zero_accum(h))) return rc;
    PushArgs a = push_args(h);
    a.step = (uint32_t)n;
    a.bin = 1;
    a.bin_only = 1;
    a.write_qind = 1;
    if ((rc = launch_push(h, a))) return rc;
    if ((rc = reduce_accum(h)) || (rc = launch_moments(h, 1))) return rc;
    if (!h->have_import) {
      if ((rc = launch_fields(h, 0))) return rc;
    } else {
      TubeArgs ta = tube_args(h, 0);
      ta.have_import = 1;  // gravity only, EAmag kept
      k_fields<<<h->ntubes, 256, (size_t)3 * max_nq(h) * sizeof(double), h->s>>>(ta);
      h->launches++;
    }
    PushArgs p = push_args(h);
    p.step = (uint32_t)n;
    p.prologue = 1;  // interpolate at q0 (qk4 holds q0 after loading)
    p.write_qind = 1;
    p.write_qk4 = next_master || qx;
    if (qx) p.cxc = h->d_cxc;
    if ((rc = launch_push(h, p))) return rc;
    h->n = n;
    return KAOS_OK;
  }
  const bool master = is_master(h, n);
  const uint32_t nn = (uint32_t)(n / h->P.ndatfac + 1);
  // ConvectionSub runs first on a master step (_8_KineticSolver.f90:62)
  if (master && !h->pending.empty()) {
    if ((rc = apply_pending_tubes(h))) return rc;
    for (auto &pt : h->pending) h->applied.push_back(std::move(pt));
    h->pending.clear();
  }
  // an idle interval converts nothing: no selection; its master step still
  // counts Qindk1 for the next interval, into rows cleared here
  const bool cx_on = qx && !h->cx_idle;
  if (cx_on && (rc = launch_cx(h))) return rc;
  if (qx && !cx_on && master)
    CK(cudaMemsetAsync(h->d_cxc, 0, (size_t)h->ncx * max_nq(h) * sizeof(unsigned), h->s));
  if (master) {
    const int compact = bc_decide(h, n);
    if ((rc = launch_boundary(h, compact))) return rc;
    bc_after(h, compact);
    if (qx && (rc = launch_boundary_ena(h))) return rc;
    if ((rc = launch_fields(h, 1))) return rc;
    if ((rc = zero_accum(h))) return rc;
  }
  PushArgs p = push_args(h);
  p.step = (uint32_t)n;
  p.bin = master;
  p.prologue = master;
  const bool cx_rec = cx_on || (qx && master);  // state the selection reads
  p.write_qind = (!h->mixed) || next_master || cx_rec || h->export_on;
  p.write_qk4 = next_master || cx_rec;
  if (cx_rec) p.cxc = h->d_cxc;
  // the ENA push (independent of the ions) runs beside the ion push
  if (cx_on && (rc = launch_push_ena(h, master))) return rc;
  if ((rc = launch_push(h, p))) return rc;
  if (cx_on && (rc = join_push_ena(h))) return rc;
  if (master) {
    if (h->P.LBCONDITIONflag == 1 && (rc = launch_inject(h, 0))) return rc;
    if (h->P.UBCONDITIONflag == 1 && (rc = launch_inject(h, 1))) return rc;
    if ((rc = reduce_accum(h)) || (rc = launch_moments(h, nn))) return rc;
  }
  h->n = n;
  return KAOS_OK;
}

// Launch-shape autotuner: the live ion state is copied into the spare
// buffer set and the push of the next step is timed there for every
// candidate (ions per work item x one block per item or a persistent grid);
// the fastest is kept.  The simulation state is not touched, and results do
// not depend on the choice (every ion is pushed by the same code).
int autotune(kaos_handle *h) {
  const int other = 1 - h->cur;
  const Fields F = ion_fields(h, h->cur, other);
  for (int f = 0; f < F.n; ++f)
    CK(cudaMemcpyAsync(F.f[f].dst, F.f[f].src, (size_t)h->ion_len * F.f[f].size,
                       cudaMemcpyDeviceToDevice, h->s));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  float best = 1e30f;
  int bw = h->wsel, bp = h->persistent, br = h->regsel;
  for (int m = 0; m < NCHUNKS; ++m)
    for (int pm = 0; pm < 2; ++pm)
    for (int rs = 0; rs < (h->mixed ? 3 : 1); ++rs) {
      h->wsel = m;
      h->persistent = pm;
      h->regsel = rs;
      PushArgs a = push_args(h);
      a.ion = h->ion[other];
      a.step = (uint32_t)(h->n + 1);
      a.write_qind = 1;
      a.write_qk4 = 0;
      float tmin = 1e30f;
      for (int rep = 0; rep < 3; ++rep) {  // the first is a warm-up
        CK(cudaEventRecord(e0, h->s));
        const int npev0 = h->npev;
        const int64_t l0 = h->launches;
        int rc = launch_push(h, a);
        h->npev = npev0;   // tuning pushes are not part of the step timing
        h->launches = l0;
        if (rc) return rc;
        CK(cudaEventRecord(e1, h->s));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        if (rep > 0) tmin = std::min(tmin, ms);
      }
      if (tmin < best) { best = tmin; bw = m; bp = pm; br = rs; }
    }
  h->wsel = bw;
  h->persistent = bp;
  h->regsel = br;
  // the master-step variant (field re-interpolation and binning) has its
  // own register needs: its budget is timed separately with the chosen
  // work-item shape (the binning accumulators it fills are cleared before
  // the next master step uses them)
  int bm = br;
  if (h->mixed) {
    float bestm = 1e30f;
    for (int rs = 0; rs < 3; ++rs) {
      h->regsel_master = rs;
      PushArgs a = push_args(h);
      a.ion = h->ion[other];
      a.step = (uint32_t)(h->n + 1);
      a.write_qind = 1;
      a.bin = 1;
      a.prologue = 1;
      float tmin = 1e30f;
      for (int rep = 0; rep < 3; ++rep) {
        CK(cudaEventRecord(e0, h->s));
        const int npev0 = h->npev;
        const int64_t l0 = h->launches;
        int rc = launch_push(h, a);
        h->npev = npev0;
        h->launches = l0;
        if (rc) return rc;
        CK(cudaEventRecord(e1, h->s));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        if (rep > 0) tmin = std::min(tmin, ms);
      }
      if (tmin < bestm) { bestm = tmin; bm = rs; }
    }
  }
  h->regsel_master = bm;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  h->tune_pending = 0;
  for (auto &g : h->graphs) cudaGraphExecDestroy(g.second.exec);
  h->graphs.clear();
  return KAOS_OK;
}

// Steps of one kind replayed from a cached CUDA graph.  A graph holds g
// consecutive steps that share their launch sequence; its key is what the
// sequence depends on: g, master / next-master step, the current ion and ENA
// buffers (the compaction alternates them) and the export switch.  The first
// use captures the steps (which advances the host state as an eager step
// does); a replay applies the same host-side transitions.
int graph_steps(kaos_handle *h, int g) {
  const int64_t n = h->n + 1;
  // a master step is replayed alone; whether it compacts is decided first
  const int compact = is_master(h, n) ? bc_decide(h, n) : 0;
  const uint64_t key = (uint64_t)g | ((uint64_t)is_master(h, n) << 16) |
                       ((uint64_t)compact << 21) |
                       ((uint64_t)is_master(h, n + 1) << 17) |
                       ((uint64_t)h->cur << 18) | ((uint64_t)h->ecur << 19) |
                       ((uint64_t)(h->export_on != 0) << 20) |
                       ((uint64_t)(h->cx_idle != 0) << 22);
  if (!h->dstep_valid) {
    k_set_step<<<1, 1, 0, h->s>>>(h->d_step, (uint32_t)h->n);
    h->launches++;
    CK(cudaGetLastError());
    h->dstep_valid = 1;
  }
  auto it = h->graphs.find(key);
  if (it != h->graphs.end()) {
    CK(cudaGraphLaunch(it->second.exec, h->s));
    h->launches += it->second.launches;
    for (int k = 0; k < g; ++k) {
      const int64_t m = h->n + 1;
      if (is_master(h, m)) {  // launch_boundary / launch_boundary_ena swaps
        bc_after(h, bc_decide(h, m));
        if (h->P.QEXCHANGEflag == 1) {
          h->ecur = 1 - h->ecur;
          h->cx_stat_pending = 1;  // the graph copied the next interval's stat
        }
      }
      h->n = m;
    }
    return KAOS_OK;
  }
  kaos_handle::StepGraph sg;
  const int64_t l0 = h->launches;
  CK(cudaStreamBeginCapture(h->s, cudaStreamCaptureModeThreadLocal));
  h->capturing = 1;
  int rc = KAOS_OK;
  for (int k = 0; k < g && rc == KAOS_OK; ++k) rc = step_once(h);
  h->capturing = 0;
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(h->s, &graph);
  if (rc != KAOS_OK) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (ce != cudaSuccess)
    return fail(h, KAOS_ERR_CUDA, "step capture: %s", cudaGetErrorString(ce));
  const cudaError_t ie = cudaGraphInstantiate(&sg.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess)
    return fail(h, KAOS_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ie));
  sg.launches = h->launches - l0;
  h->graphs[key] = sg;
  CK(cudaGraphLaunch(sg.exec, h->s));
  return KAOS_OK;
}

constexpr int GRAPH_RUN = 8;  // ordinary steps per replayed graph

}  // namespace

// ===========================================================================
extern "C" {

const char *kaos_version(void) { return "kaos_b200 0.1.0 (sm_100a)"; }

const char *kaos_last_error(kaos_handle *h) {
  return h ? h->err : "null handle";
}

int kaos_create(const kaos_params_c *p, const kaos_tube_c *tubes,
                int32_t ntubes, const kaos_vgrid_c *vgc, kaos_handle **out) {
  if (!p || !tubes || !vgc || !out || ntubes < 1) return KAOS_ERR_PARAM;
  if (p->QEXCHANGEflag == 1 && ntubes > KAOS_MAX_TUBES_CX) return KAOS_ERR_PARAM;
  *out = nullptr;
  kaos_handle *h = new kaos_handle();
  h->P = *p;
  if (h->P.ndatfac < 1) h->P.ndatfac = 1;
  if (h->P.h <= 0.0 || h->P.ms <= 0.0) {
    int rc = fail(h, KAOS_ERR_PARAM, "h and ms must be positive");
    *out = h;
    return rc;
  }
  if (p->precision != KAOS_PREC_FP64 && p->precision != KAOS_PREC_MIXED &&
      p->precision != KAOS_PREC_MIXED_K64) {
    *out = h;
    return fail(h, KAOS_ERR_PARAM, "unknown precision mode %d", (int)p->precision);
  }
  h->mixed = p->precision == KAOS_PREC_MIXED || p->precision == KAOS_PREC_MIXED_K64;
  h->kick64 = p->precision == KAOS_PREC_MIXED_K64;
  h->three_d = p->ION2VPERPflag == 1;
  h->ntubes = ntubes;
  h->id_base.assign(ntubes, 0);
  VGridC &vg = h->vg;
  vg.three_d = h->three_d;
  vg.n1 = vgc->n1;
  vg.n2 = h->three_d ? vgc->n2 : 0;
  vg.npar = vgc->npar;
  if (vg.n1 < 1 || vg.npar < 1 || vg.n1 > MAXV || vg.npar > MAXV ||
      (h->three_d && (vg.n2 < 1 || vg.n2 > MAXV)) || !vgc->e1 || !vgc->epar ||
      (h->three_d && !vgc->e2)) {
    *out = h;
    return fail(h, KAOS_ERR_PARAM, "velocity grid sizes must be in [1, %d]", MAXV);
  }
  for (int k = 0; k <= vg.n1; ++k) { vg.e1[k] = vgc->e1[k]; vg.f1[k] = (float)vgc->e1[k]; }
  for (int k = 0; k <= vg.npar; ++k) { vg.epar[k] = vgc->epar[k]; vg.fpar[k] = (float)vgc->epar[k]; }
  for (int k = 0; h->three_d && k <= vg.n2; ++k) { vg.e2[k] = vgc->e2[k]; vg.f2[k] = (float)vgc->e2[k]; }
  h->nv = h->three_d ? vg.n1 * vg.n2 * vg.npar : vg.n1 * vg.npar;
  // ENA grid until kaos_set_ena_grid: Vp <- Vperp1 axis, Vq <- Vpar axis,
  // Vphi <- Vperp2 axis (Vperp1 on a 2D ion grid)
  h->evg = vg;
  h->evg.three_d = 1;
  if (!h->three_d) {
    h->evg.n2 = vg.n1;
    for (int k = 0; k <= vg.n1; ++k) { h->evg.e2[k] = vg.e1[k]; h->evg.f2[k] = vg.f1[k]; }
  }

  // ---- tubes: descriptors, concatenated per-cell tables -----------------
  std::vector<double> qGL, qGH, qGC, hqC, dqC, d3xC, rGC, thC, elC, TeG, TsG,
      neut, lam, eta, xi1, xi2, S0, Om0, chi1, chi2, uL, uH, hK1, hK2, hc1,
      hc2, hiom0, uM;
  int64_t poff = 0, coff = 0, moff = 0, hoff = 0, eoff = 0;
  for (int t = 0; t < ntubes; ++t) {
    const kaos_tube_c &T = tubes[t];
    if (T.nq < 6 || T.nq > MAX_CELLS || T.capacity < 1 || !T.qGL || !T.qGH ||
        !T.qGC || !T.hqC || !T.dqC || !T.d3xC || !T.rGC || !T.thetaGC ||
        !T.ellGC || !T.TeG || !T.TsG) {
      *out = h;
      return fail(h, KAOS_ERR_PARAM, "tube %d: nq must be in [6, %d], capacity > 0, tables non-NULL", t, MAX_CELLS);
    }
    // MomentFilterSub (_8_7_1_MomentFilter.f90:30-142) reads Pt cells around
    // each cell; a tube shorter than the window would read outside it
    if (p->MOMENTFILTERflag == 1) {
      const int pts[5] = {p->M0MAfilterPt, p->M1ParMAfilterPt, p->M1Perp1MAfilterPt,
                          p->M1Perp2MAfilterPt, p->M2ParMAfilterPt};
      for (int w : pts)
        if (w < 3 || w % 2 == 0 || T.nq < w) {
          *out = h;
          return fail(h, KAOS_ERR_PARAM,
                      "tube %d: moving-average windows must be odd, >= 3 and at most nq (%d): got %d",
                      t, T.nq, w);
        }
    }
    for (int k = 0; k + 1 < T.nq; ++k)
      if (T.qGH[k] != T.qGL[k + 1]) {
        *out = h;
        return fail(h, KAOS_ERR_PARAM, "tube %d: cells must be contiguous (qGH[%d] != qGL[%d])", t, k, k + 1);
      }
    TubeD d{};
    d.nq = T.nq;
    d.coff = (int)coff;
    d.off = poff;
    d.cap = T.capacity;
    d.pG = T.pG;
    d.phiG = T.phiG;
    d.cphi = std::cos(T.phiG);
    d.sphi = std::sin(T.phiG);
    d.sgn = (T.qGL[0] <= 0.0) ? 1.0 : -1.0;
    d.nsnormfac = T.nsnormfac;
    d.nsnormCLB = T.nsnormCLB;
    d.nsnormCUB = T.nsnormCUB;
    d.sumdsICR = T.sumdsICR;
    d.ms = T.ms > 0.0 ? T.ms : p->ms;
    d.qs = T.qs != 0.0 ? T.qs : p->qs;
    d.moff = moff;
    d.hoff = hoff;
    d.ecap = (p->QEXCHANGEflag == 1) ? (int64_t)T.capacity / 4 + 4096 : 0;
    d.eoff = eoff;
    eoff += d.ecap;
    host_rho_z(T.qGC[0], T.pG, &d.rhoLB, &d.zLB);
    host_rho_z(T.qGC[T.nq - 1], T.pG, &d.rhoUB, &d.zUB);
    h->th.push_back(d);
    auto app = [&](std::vector<double> &v, const double *src, double dflt) {
      for (int k = 0; k < T.nq; ++k) v.push_back(src ? src[k] : dflt);
    };
    app(qGL, T.qGL, 0); app(qGH, T.qGH, 0); app(qGC, T.qGC, 0);
    app(hqC, T.hqC, 0); app(dqC, T.dqC, 0); app(d3xC, T.d3xC, 1);
    app(rGC, T.rGC, 0); app(thC, T.thetaGC, 0); app(elC, T.ellGC, 1);
    app(TeG, T.TeG, 0); app(TsG, T.TsG, 0); app(neut, T.nsnormCNeut, 0);
    app(lam, T.lambdaPerp, 0); app(eta, T.EtaLH, 0); app(xi1, T.XiPerp1, 0);
    app(xi2, T.XiPerp2, 0); app(S0, T.S0, 0); app(Om0, T.OmegaG0, 1);
    app(chi1, T.ChiPerp1, 0); app(chi2, T.ChiPerp2, 0);
    // wave-heating constants: K_i = h sqrt(q^2 xi_i eta S0 / (2 m^2 pi))
    for (int k = 0; k < T.nq; ++k) {
      const double pre = (d.qs * d.qs / (2.0 * d.ms * d.ms)) *
                         (T.S0 ? T.S0[k] : 0.0) * (T.EtaLH ? T.EtaLH[k] : 0.0);
      hK1.push_back(p->h * std::sqrt(pre * (T.XiPerp1 ? T.XiPerp1[k] : 0.0) / PI));
      hK2.push_back(p->h * std::sqrt(pre * (T.XiPerp2 ? T.XiPerp2[k] : 0.0) / PI));
      hc1.push_back(0.5 * (T.ChiPerp1 ? T.ChiPerp1[k] : 0.0));
      hc2.push_back(0.5 * (T.ChiPerp2 ? T.ChiPerp2[k] : 0.0));
      hiom0.push_back(T.OmegaG0 && T.OmegaG0[k] != 0.0 ? 1.0 / T.OmegaG0[k] : 0.0);
    }
    for (int k = 0; k < T.nq; ++k) {
      uL.push_back(host_quartic_u(T.qGL[k], T.pG));
      uH.push_back(host_quartic_u(T.qGH[k], T.pG));
      uM.push_back(host_quartic_u(0.5 * (T.qGL[k] + T.qGH[k]), T.pG));
    }
    poff += T.capacity;
    coff += T.nq;
    moff += T.nq;
    hoff += (int64_t)T.nq * h->nv;
  }
  h->ncell = coff;
  h->bc_bound.assign(ntubes, 0);
  *out = h;
  int rc;
  CK(cudaStreamCreateWithFlags(&h->s, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&h->s2, cudaStreamNonBlocking));
  CK(cudaEventCreate(&h->e0));
  CK(cudaEventCreate(&h->e1));
  CK(cudaEventCreateWithFlags(&h->efork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&h->ejoin, cudaEventDisableTiming));
  CellTables &c = h->ct;
  c.ncell_total = coff;
  double *tmp;
#define UP(field, vec)                                  \
  if ((rc = upload(h, &tmp, vec))) return rc;           \
  c.field = tmp;
  UP(qGL, qGL) UP(qGH, qGH) UP(qGC, qGC) UP(hqC, hqC) UP(dqC, dqC)
  UP(d3xC, d3xC) UP(rGC, rGC) UP(thetaGC, thC) UP(ellGC, elC) UP(TeG, TeG)
  UP(TsG, TsG) UP(nsnormCNeut, neut) UP(lambdaPerp, lam) UP(EtaLH, eta)
  UP(XiPerp1, xi1) UP(XiPerp2, xi2) UP(S0, S0) UP(OmegaG0, Om0)
  UP(ChiPerp1, chi1) UP(ChiPerp2, chi2) UP(uL, uL) UP(uH, uH)
  UP(hK1, hK1) UP(hK2, hK2) UP(hc1, hc1) UP(hc2, hc2) UP(hiom0, hiom0) UP(uM, uM)
  UP(Te, TeG)
#undef UP
  if ((rc = dalloc(h, &c.EAmag, coff))) return rc;
  if ((rc = dalloc(h, &c.EG, coff))) return rc;
  if ((rc = dalloc(h, &c.M0prev, coff))) return rc;
  if ((rc = dalloc(h, &c.nuPoi, coff))) return rc;
  if ((rc = dalloc(h, &c.mom, coff * KAOS_NMOMENTS))) return rc;
  h->host_cells = {qGL, qGH, qGC};
  // binning accumulators, ions then ENAs, in one block (one reduction
  // covers them all when a tube is split across ranks)
  {
    const size_t nc = (size_t)coff;
    const size_t ion_n = nc * (1 + vg.npar + vg.n1 + std::max(vg.n2, 1));
    const size_t ena_n = p->QEXCHANGEflag == 1 ? nc * (1 + 3 * (size_t)MAXV) : 0;
    unsigned *base = nullptr;
    if ((rc = dalloc(h, &base, ion_n + ena_n))) return rc;
    h->acc_base = base;
    h->acc_len = (int64_t)(ion_n + ena_n);
    h->acc.cnt = base;
    h->acc.mpar = base + nc;
    h->acc.m1 = h->acc.mpar + nc * vg.npar;
    h->acc.m2 = h->acc.m1 + nc * vg.n1;
    if (ena_n) {
      h->acc.ecnt = base + ion_n;
      h->acc.emp = h->acc.ecnt + nc;
      h->acc.emq = h->acc.emp + nc * MAXV;
      h->acc.emph = h->acc.emq + nc * MAXV;
    }
  }
  // tube descriptors and the static block -> (tube, chunk) map
  std::vector<int> bt;
  std::vector<int64_t> bs;
  const int64_t chunk = PUSH_THREADS * PUSH_ITEMS;
  for (int t = 0; t < ntubes; ++t) {
    h->tube_blk0.push_back((int)bt.size());
    for (int64_t s0 = 0; s0 < h->th[t].cap; s0 += chunk) {
      bt.push_back(t);
      bs.push_back(s0);
    }
  }
  h->tube_blk0.push_back((int)bt.size());
  h->nblk = (int)bt.size();
  if ((rc = dalloc(h, &h->d_tubes, ntubes))) return rc;
  CK(cudaMemcpy(h->d_tubes, h->th.data(), ntubes * sizeof(TubeD), cudaMemcpyHostToDevice));
  if ((rc = dalloc(h, &h->d_blk_tube, bt.size()))) return rc;
  if ((rc = dalloc(h, &h->d_blk_start, bs.size()))) return rc;
  if ((rc = dalloc(h, &h->d_tube_blk0, h->tube_blk0.size()))) return rc;
  CK(cudaMemcpy(h->d_blk_tube, bt.data(), bt.size() * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_blk_start, bs.data(), bs.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_tube_blk0, h->tube_blk0.data(), h->tube_blk0.size() * sizeof(int), cudaMemcpyHostToDevice));
  for (int m = 0; m < NCHUNKS; ++m) {
    std::vector<int> wt;
    std::vector<int64_t> ws;
    for (int t = 0; t < ntubes; ++t)
      for (int64_t s0 = 0; s0 < h->th[t].cap; s0 += CHUNKS[m]) {
        wt.push_back(t);
        ws.push_back(s0);
      }
    kaos_handle::WorkMap &M = h->wmap[m];
    M.chunk = CHUNKS[m];
    M.n = (int)wt.size();
    if ((rc = dalloc(h, &M.d_tube, wt.size())) || (rc = dalloc(h, &M.d_start, ws.size())))
      return rc;
    CK(cudaMemcpy(M.d_tube, wt.data(), wt.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(M.d_start, ws.data(), ws.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
  }
  if ((rc = dalloc(h, &h->d_nlive, ntubes))) return rc;
  if ((rc = dalloc(h, &h->d_nlive_new, ntubes))) return rc;
  if ((rc = dalloc(h, &h->d_next_id, ntubes))) return rc;
  if ((rc = dalloc(h, &h->d_blkcnt, bt.size()))) return rc;
  if ((rc = dalloc(h, &h->d_blkoff, bt.size()))) return rc;
  if ((rc = dalloc(h, &h->d_lb_out, ntubes))) return rc;
  if ((rc = dalloc(h, &h->d_ub_out, ntubes))) return rc;
  if ((rc = dalloc(h, &h->d_lb_in, ntubes))) return rc;
  if ((rc = dalloc(h, &h->d_ub_in, ntubes))) return rc;
  if ((rc = dalloc(h, &h->d_status, 1))) return rc;
  if ((rc = dalloc(h, &h->d_step, 1))) return rc;
  // particle arrays (two buffer sets for the order-preserving compaction)
  const int64_t cap = poff;
  h->ion_len = cap;
  for (int b = 0; b < 2; ++b) {
    Ions &I = h->ion[b];
    if (h->mixed) {
      if ((rc = dalloc(h, &I.x, cap))) return rc;
      if ((rc = dalloc(h, &I.vpar, cap))) return rc;
      if ((rc = dalloc(h, &I.v12, cap))) return rc;
      if ((rc = dalloc(h, &I.ffl, cap))) return rc;
      if ((rc = dalloc(h, &I.fqk4, cap))) return rc;
    } else {
      if ((rc = dalloc(h, &I.rho, cap))) return rc;
      if ((rc = dalloc(h, &I.z, cap))) return rc;
      if ((rc = dalloc(h, &I.vpar, cap))) return rc;
      if ((rc = dalloc(h, &I.v1, cap))) return rc;
      if ((rc = dalloc(h, &I.v2, cap))) return rc;
      if ((rc = dalloc(h, &I.aea, cap))) return rc;
      if ((rc = dalloc(h, &I.ag, cap))) return rc;
      if ((rc = dalloc(h, &I.qk4, cap))) return rc;
      if (p->QEXCHANGEflag == 1) {
        if ((rc = dalloc(h, &I.rho4, cap))) return rc;
        if ((rc = dalloc(h, &I.z4, cap))) return rc;
      }
    }
    if ((rc = dalloc(h, &I.qind, cap))) return rc;
    if (!h->three_d && (rc = dalloc(h, &I.vb, cap))) return rc;
    if ((rc = dalloc(h, &I.id, cap))) return rc;
  }
  // global cell -> (tube, cell) map
  {
    std::vector<int> ctb, cq;
    for (int t = 0; t < ntubes; ++t)
      for (int k = 0; k < h->th[t].nq; ++k) { ctb.push_back(t); cq.push_back(k); }
    if ((rc = dalloc(h, &h->d_cell_tube, ctb.size())) || (rc = dalloc(h, &h->d_cell_q, cq.size())))
      return rc;
    CK(cudaMemcpy(h->d_cell_tube, ctb.data(), ctb.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->d_cell_q, cq.data(), cq.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  // ENA arrays, block map and charge-exchange chunk map
  if (p->QEXCHANGEflag == 1) {
    const int64_t ecap_all = eoff;
    for (int b = 0; b < 2; ++b) {
      Enas &E = h->ena[b];
      if ((rc = dalloc(h, &E.x, ecap_all)) || (rc = dalloc(h, &E.y, ecap_all)) ||
          (rc = dalloc(h, &E.z, ecap_all)) || (rc = dalloc(h, &E.vx, ecap_all)) ||
          (rc = dalloc(h, &E.vy, ecap_all)) || (rc = dalloc(h, &E.vz, ecap_all)) ||
          (rc = dalloc(h, &E.vps, ecap_all)) || (rc = dalloc(h, &E.vphs, ecap_all)) ||
          (rc = dalloc(h, &E.qind, ecap_all)) || (rc = dalloc(h, &E.vb, ecap_all)) ||
          (rc = dalloc(h, &E.id, ecap_all)))
        return rc;
    }
    std::vector<int> ebt, te0, cxt, tc0;
    std::vector<int64_t> ebs, cxs;
    for (int t = 0; t < ntubes; ++t) {
      te0.push_back((int)ebt.size());
      for (int64_t s0 = 0; s0 < h->th[t].ecap; s0 += chunk) {
        ebt.push_back(t);
        ebs.push_back(s0);
      }
      tc0.push_back((int)cxt.size());
      for (int64_t s0 = 0; s0 < h->th[t].cap; s0 += CX_CHUNK) {
        cxt.push_back(t);
        cxs.push_back(s0);
      }
    }
    te0.push_back((int)ebt.size());
    tc0.push_back((int)cxt.size());
    h->neblk = (int)ebt.size();
    h->ncx = (int)cxt.size();
    auto up_i = [&](int **d, const std::vector<int> &v) {
      int r = dalloc(h, d, v.size());
      if (!r && cudaMemcpy(*d, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
        r = fail(h, KAOS_ERR_CUDA, "upload failed");
      return r;
    };
    auto up_l = [&](int64_t **d, const std::vector<int64_t> &v) {
      int r = dalloc(h, d, v.size());
      if (!r && cudaMemcpy(*d, v.data(), v.size() * sizeof(int64_t), cudaMemcpyHostToDevice) != cudaSuccess)
        r = fail(h, KAOS_ERR_CUDA, "upload failed");
      return r;
    };
    if ((rc = up_i(&h->d_eblk_tube, ebt)) || (rc = up_l(&h->d_eblk_start, ebs)) ||
        (rc = up_i(&h->d_tube_eblk0, te0)) || (rc = up_i(&h->d_cx_tube, cxt)) ||
        (rc = up_l(&h->d_cx_start, cxs)) || (rc = up_i(&h->d_tube_cx0, tc0)))
      return rc;
    if ((rc = dalloc(h, &h->d_nena, ntubes)) || (rc = dalloc(h, &h->d_nena_new, ntubes)) ||
        (rc = dalloc(h, &h->d_eblkcnt, ebt.size())) || (rc = dalloc(h, &h->d_eblkoff, ebt.size())) ||
        (rc = dalloc(h, &h->d_lbe_out, ntubes)) || (rc = dalloc(h, &h->d_ube_out, ntubes)) ||
        (rc = dalloc(h, &h->d_cxconv, cxt.size())) ||
        (rc = dalloc(h, &h->d_cxbase, cxt.size())) ||
        (rc = dalloc(h, &h->d_cxend, (size_t)h->ncell)) ||
        (rc = dalloc(h, &h->d_tube_done, (size_t)ntubes)) ||
        (rc = dalloc(h, &h->d_cx_list, (size_t)h->ncell)) ||
        (rc = dalloc(h, &h->d_cx_nlist, 1)) ||
        (rc = dalloc(h, &h->d_cx_chunks, cxt.size())) ||
        (rc = dalloc(h, &h->d_cx_nchunk, 2)) ||
        (rc = dalloc(h, &h->d_tube_active, (size_t)ntubes)) ||
        (rc = dalloc(h, &h->d_cxc, cxt.size() * (size_t)max_nq(h))) ||
        (rc = dalloc(h, &h->d_cxo, cxt.size() * (size_t)max_nq(h))))
      return rc;
    CK(cudaMallocHost((void **)&h->cx_stat, (size_t)(ntubes + 1) * sizeof(int64_t)));
    memset(h->cx_stat, 0, (size_t)(ntubes + 1) * sizeof(int64_t));
  }
  // kernels whose per-tube shared tables may exceed the default 48 KB
  {
    const size_t nq = (size_t)max_nq(h);
    const std::pair<const void *, size_t> big[] = {
        {(const void *)k_collision_counts, 8 * nq * sizeof(double)},
        {(const void *)k_cx_convert, cx_convert_smem((int)nq)},
        {(const void *)k_fields, 3 * nq * sizeof(double)},
        {(const void *)k_push_ena, ena_push_smem((int)nq, ntubes)},
        {(const void *)k_load, (nq + 1) * sizeof(double)}};
    for (const auto &b : big)
      if (b.second > 48 * 1024)
        CK(cudaFuncSetAttribute(b.first, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b.second));
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cx_convert, 256,
                                                     cx_convert_smem((int)nq)));
    h->cx_blocks = std::max(1, per_sm) * sm_count(h);
  }
  CK(cudaDeviceSynchronize());
  return KAOS_OK;
}

int kaos_load_particles(kaos_handle *h, int32_t tube, const double *q,
                        const double *vpar, const double *vperp1,
                        const double *vperp2, int64_t n) {
  if (!h) return KAOS_ERR_PARAM;
  if (tube < 0 || tube >= h->ntubes) return fail(h, KAOS_ERR_PARAM, "bad tube %d", tube);
  if (!q || !vpar || !vperp1 || n < 0) return fail(h, KAOS_ERR_PARAM, "null input");
  if (h->n != 0) return fail(h, KAOS_ERR_STATE, "particles must be loaded before the first step");
  const TubeD &T = h->th[tube];
  if (n > T.cap) return fail(h, KAOS_ERR_CAPACITY, "tube %d: %lld particles exceed capacity %lld", tube, (long long)n, (long long)T.cap);
  if (n > 0) {
    // the caller's arrays go to the spare buffer set (no allocation); k_load
    // derives the per-ion state from there (clamp, cell search, bins,
    // positions)
    const int na = vperp2 ? 4 : 3;
    double *stage[4];
    spare_slots(h, tube, stage, nullptr);
    const double *src[4] = {q, vpar, vperp1, vperp2};
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < na && e == cudaSuccess; ++k)
      e = cudaMemcpy(stage[k], src[k], n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_vg, &h->vg, sizeof(VGridC));
    g_grid_owner = nullptr;  // c_evg may belong to another handle
    if (e == cudaSuccess) {
      LoadArgs a{};
      a.T = T;
      a.q = stage[0];
      a.vpar = stage[1];
      a.v1 = stage[2];
      a.v2 = vperp2 ? stage[3] : nullptr;
      a.n = n;
      a.id0 = h->id_base[tube];
      a.ion = h->ion[h->cur];
      a.ct = h->ct;
      a.mixed = h->mixed;
      const int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 32);
      k_load<<<grid, 256, (size_t)(T.nq + 1) * sizeof(double)>>>(a);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return fail(h, KAOS_ERR_CUDA, "load: %s", cudaGetErrorString(e));
  }
  int64_t nl = n;
  uint64_t nid = h->id_base[tube] + (uint64_t)n;
  h->bc_bound[tube] = n;
  CK(cudaMemcpy(h->d_nlive + tube, &nl, sizeof(int64_t), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_next_id + tube, &nid, sizeof(uint64_t), cudaMemcpyHostToDevice));
  if (h->d_cxc)  // the first push starts the selection counts from zero
    CK(cudaMemset(h->d_cxc, 0, (size_t)h->ncx * max_nq(h) * sizeof(unsigned)));
  h->loaded = 1;
  return KAOS_OK;
}

int kaos_init_particles(kaos_handle *h, int32_t tube, const kaos_init_c *in) {
  if (!h) return KAOS_ERR_PARAM;
  if (tube < 0 || tube >= h->ntubes) return fail(h, KAOS_ERR_PARAM, "bad tube %d", tube);
  if (!in || !in->counts) return fail(h, KAOS_ERR_PARAM, "null counts");
  if (h->n != 0) return fail(h, KAOS_ERR_STATE, "particles must be loaded before the first step");
  const TubeD &T = h->th[tube];
  const int nu = (int)std::llround(2.0 * in->kappa - 1.0);
  if (!(in->tail_fraction >= 0.0 && in->tail_fraction <= 1.0) ||
      (in->tail_fraction > 0.0 &&
       (std::fabs(2.0 * in->kappa - 1.0 - nu) > 1e-9 || nu < 3 || nu > 63 || !(in->tail_T > 0.0))))
    return fail(h, KAOS_ERR_PARAM, "init: tail_fraction in [0,1]; 2 kappa - 1 an integer in [3, 63]; tail_T > 0");
  std::vector<int64_t> pre(T.nq + 1, 0);
  for (int k = 0; k < T.nq; ++k) {
    if (in->counts[k] < 0) return fail(h, KAOS_ERR_PARAM, "negative count in cell %d", k);
    pre[k + 1] = pre[k] + in->counts[k];
  }
  const int64_t n = pre[T.nq];
  if (n > T.cap) return fail(h, KAOS_ERR_CAPACITY, "tube %d: %lld particles exceed capacity %lld", tube, (long long)n, (long long)T.cap);
  int64_t *d_pre = nullptr;
  if (cudaMalloc(&d_pre, pre.size() * sizeof(int64_t)) != cudaSuccess)
    return fail(h, KAOS_ERR_CUDA, "cudaMalloc of the init prefix failed");
  InitArgs a{};
  a.T = T;
  a.pre = d_pre;
  a.n = n;
  a.id0 = h->id_base[tube];
  a.ion = h->ion[h->cur];
  a.ct = h->ct;
  a.tail_fraction = in->tail_fraction;
  a.nu = nu;
  a.s_tail = in->tail_fraction > 0.0
                 ? std::sqrt(KB * in->tail_T / T.ms * (double)(nu - 2) / (double)nu) : 0.0;
  a.seed = in->seed;
  a.mixed = h->mixed;
  cudaError_t e = cudaMemcpy(d_pre, pre.data(), pre.size() * sizeof(int64_t), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_vg, &h->vg, sizeof(VGridC));
    g_grid_owner = nullptr;  // c_evg may belong to another handle
  if (e == cudaSuccess && n > 0) {
    const int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 32);
    k_init<<<grid, 256>>>(a);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  cudaFree(d_pre);
  if (e != cudaSuccess) return fail(h, KAOS_ERR_CUDA, "init: %s", cudaGetErrorString(e));
  int64_t nl = n;
  uint64_t nid = h->id_base[tube] + (uint64_t)n;
  h->bc_bound[tube] = n;
  CK(cudaMemcpy(h->d_nlive + tube, &nl, sizeof(int64_t), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_next_id + tube, &nid, sizeof(uint64_t), cudaMemcpyHostToDevice));
  if (h->d_cxc)  // the first push starts the selection counts from zero
    CK(cudaMemset(h->d_cxc, 0, (size_t)h->ncx * max_nq(h) * sizeof(unsigned)));
  h->loaded = 1;
  return KAOS_OK;
}

int kaos_set_fields(kaos_handle *h, int32_t tube, const double *EAmag,
                    int32_t nq) {
  if (!h) return KAOS_ERR_PARAM;
  if (tube < 0 || tube >= h->ntubes) return fail(h, KAOS_ERR_PARAM, "bad tube %d", tube);
  if (!EAmag) {
    h->have_import = 0;
    return KAOS_OK;
  }
  if (nq != h->th[tube].nq) return fail(h, KAOS_ERR_PARAM, "nq mismatch");
  CK(cudaMemcpy(h->ct.EAmag + h->th[tube].coff, EAmag, nq * sizeof(double), cudaMemcpyHostToDevice));
  h->have_import = 1;
  return KAOS_OK;
}

int kaos_set_export(kaos_handle *h, int32_t on) {
  if (!h) return KAOS_ERR_PARAM;
  if (on && !h->acc.hist) {
    int rc = dalloc(h, &h->acc.hist, (size_t)h->ncell * h->nv);
    if (rc) return rc;
  }
  h->export_on = on ? 1 : 0;
  return KAOS_OK;
}

int kaos_set_graph(kaos_handle *h, int32_t on) {
  if (!h) return KAOS_ERR_PARAM;
  h->graph = on ? 1 : 0;
  return KAOS_OK;
}

int kaos_set_launch(kaos_handle *h, int32_t chunk, int32_t mode) {
  if (!h) return KAOS_ERR_PARAM;
  if (chunk == 0 || mode < 0) {
    h->tune_pending = 1;
    return KAOS_OK;
  }
  int m = -1;
  for (int k = 0; k < NCHUNKS; ++k)
    if (CHUNKS[k] == chunk) m = k;
  if (m < 0 || mode > 31 || ((mode >> 1) & 3) == 3)
    return fail(h, KAOS_ERR_PARAM, "launch: chunk must be 1024, 2048 or 4096; mode bits "
                "1-2 in 0..2, bits 3-4 in 0..3");
  h->wsel = m;
  h->persistent = mode & 1;
  h->regsel = (mode >> 1) & 3;
  h->regsel_master = ((mode >> 3) & 3) ? ((mode >> 3) & 3) - 1 : h->regsel;
  h->tune_pending = 0;
  for (auto &g : h->graphs) cudaGraphExecDestroy(g.second.exec);
  h->graphs.clear();
  return KAOS_OK;
}

int kaos_set_ena_grid(kaos_handle *h, const kaos_vgrid_c *vg) {
  if (!h || !vg) return KAOS_ERR_PARAM;
  g_grid_owner = nullptr;  // the next step uploads the new grid
  if (h->n != 0) return fail(h, KAOS_ERR_STATE, "the ENA grid is set before the first step");
  if (vg->n1 < 1 || vg->n2 < 1 || vg->npar < 1 || vg->n1 > MAXV || vg->n2 > MAXV ||
      vg->npar > MAXV || !vg->e1 || !vg->e2 || !vg->epar)
    return fail(h, KAOS_ERR_PARAM, "ENA grid sizes must be in [1, %d]", MAXV);
  VGridC &g = h->evg;
  g.three_d = 1;
  g.n1 = vg->n1;
  g.n2 = vg->n2;
  g.npar = vg->npar;
  for (int k = 0; k <= g.n1; ++k) { g.e1[k] = vg->e1[k]; g.f1[k] = (float)vg->e1[k]; }
  for (int k = 0; k <= g.n2; ++k) { g.e2[k] = vg->e2[k]; g.f2[k] = (float)vg->e2[k]; }
  for (int k = 0; k <= g.npar; ++k) { g.epar[k] = vg->epar[k]; g.fpar[k] = (float)vg->epar[k]; }
  return KAOS_OK;
}

int kaos_update_tube(kaos_handle *h, int32_t tube, const kaos_tube_c *T) {
  if (!h || !T || tube < 0 || tube >= h->ntubes) return KAOS_ERR_PARAM;
  const TubeD &cur = h->th[tube];
  if (T->nq != cur.nq || !T->qGL || !T->qGH || !T->qGC || !T->hqC || !T->dqC ||
      !T->d3xC || !T->rGC || !T->thetaGC || !T->ellGC || !T->TeG || !T->TsG)
    return fail(h, KAOS_ERR_PARAM, "tube %d: update needs the same nq and non-NULL tables", tube);
  const double *qGL = h->host_cells[0].data() + cur.coff;
  const double *qGH = h->host_cells[1].data() + cur.coff;
  for (int k = 0; k < cur.nq; ++k)
    if (T->qGL[k] != qGL[k] || T->qGH[k] != qGH[k])
      return fail(h, KAOS_ERR_PARAM, "tube %d: the q grid must stay the same (cell %d)", tube, k);
  kaos_handle::PendingTube pt;
  pt.tube = tube;
  pt.d = cur;
  pt.d.pG = T->pG;
  pt.d.phiG = T->phiG;
  pt.d.cphi = std::cos(T->phiG);
  pt.d.sphi = std::sin(T->phiG);
  pt.d.nsnormfac = T->nsnormfac;
  pt.d.nsnormCLB = T->nsnormCLB;
  pt.d.nsnormCUB = T->nsnormCUB;
  pt.d.sumdsICR = T->sumdsICR;
  host_rho_z(T->qGC[0], T->pG, &pt.d.rhoLB, &pt.d.zLB);
  host_rho_z(T->qGC[T->nq - 1], T->pG, &pt.d.rhoUB, &pt.d.zUB);
  pt.tables = tube_tables(*T, pt.d, h->P);
  for (auto &q : h->pending)
    if (q.tube == tube) {
      q = std::move(pt);
      return KAOS_OK;
    }
  h->pending.push_back(std::move(pt));
  return KAOS_OK;
}

int kaos_set_reduce(kaos_handle *h, kaos_reduce_fn fn, void *ctx) {
  if (!h) return KAOS_ERR_PARAM;
  h->reduce_fn = fn;
  h->reduce_ctx = ctx;
  return KAOS_OK;
}

int kaos_set_rank(kaos_handle *h, int32_t rank, int32_t nranks) {
  if (!h) return KAOS_ERR_PARAM;
  if (nranks < 1 || rank < 0 || rank >= nranks)
    return fail(h, KAOS_ERR_PARAM, "rank %d of %d", rank, nranks);
  h->rank = rank;
  h->nranks = nranks;
  return KAOS_OK;
}

int kaos_set_id_base(kaos_handle *h, int32_t tube, uint64_t base) {
  if (!h || tube < 0 || tube >= h->ntubes) return KAOS_ERR_PARAM;
  if (h->n != 0) return fail(h, KAOS_ERR_STATE, "ids are set before the first step");
  h->id_base[tube] = base;
  return KAOS_OK;
}

int kaos_get_launch(kaos_handle *h, int32_t *chunk, int32_t *mode) {
  if (!h || !chunk || !mode) return KAOS_ERR_PARAM;
  *chunk = CHUNKS[h->wsel];
  *mode = h->persistent | (h->regsel << 1) |
          (h->regsel_master != h->regsel ? (h->regsel_master + 1) << 3 : 0);
  return KAOS_OK;
}

int kaos_step(kaos_handle *h, int64_t nsteps) {
  if (!h) return KAOS_ERR_PARAM;
  if (!h->loaded) return fail(h, KAOS_ERR_STATE, "kaos_step before kaos_load_particles");
  if (nsteps < 0) return fail(h, KAOS_ERR_PARAM, "nsteps < 0");
  if (g_grid_owner != h) {  // the velocity grids in constant memory
    CK(cudaMemcpyToSymbolAsync(c_vg, &h->vg, sizeof(VGridC), 0, cudaMemcpyHostToDevice, h->s));
    CK(cudaMemcpyToSymbolAsync(c_evg, &h->evg, sizeof(VGridC), 0, cudaMemcpyHostToDevice, h->s));
    g_grid_owner = h;
  }
  h->launches = 0;
  h->npev = 0;
  CK(cudaEventRecord(h->e0, h->s));
  for (int64_t k = 0; k < nsteps;) {
    const int64_t n = h->n + 1;
    int rc;
    if ((rc = resolve_cx_idle(h))) return rc;
    if (h->tune_pending && n >= 2 && (rc = autotune(h))) return rc;
    if (!h->graph || n == 1 || h->reduce_fn ||
        (!h->pending.empty() && is_master(h, n))) {  // host work between kernels
      if ((rc = step_once(h))) return rc;
      h->dstep_valid = 0;
      ++k;
      continue;
    }
    int g = 1;  // a run of ordinary steps (neither master nor next-master)
    if (!is_master(h, n) && !is_master(h, n + 1))
      while (g < GRAPH_RUN && k + g < nsteps && !is_master(h, n + g) &&
             !is_master(h, n + g + 1))
        ++g;
    if ((rc = graph_steps(h, g))) return rc;
    k += g;
  }
  CK(cudaEventRecord(h->e1, h->s));
  CK(cudaEventSynchronize(h->e1));
  h->applied.clear();  // their host tables have been copied
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, h->e0, h->e1));
  h->last_ms = ms;
  h->push_ms = 0.0;
  for (int k = 0; k < h->npev; ++k) {
    float m = 0.f;
    CK(cudaEventElapsedTime(&m, h->pev[2 * k], h->pev[2 * k + 1]));
    h->push_ms += m;
  }
  uint32_t st = 0;
  CK(cudaMemcpy(&st, h->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  if (st & ST_NAN) return fail(h, KAOS_ERR_NAN, "non-finite particle state on the device");
  if (st & ST_CAP) return fail(h, KAOS_ERR_CAPACITY, "tube capacity exceeded during injection");
  return KAOS_OK;
}

int kaos_get_step(kaos_handle *h, int64_t *n) {
  if (!h || !n) return KAOS_ERR_PARAM;
  *n = h->n;
  return KAOS_OK;
}

int kaos_get_status(kaos_handle *h, uint32_t *status) {
  if (!h || !status) return KAOS_ERR_PARAM;
  CK(cudaMemcpy(status, h->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  return KAOS_OK;
}

int kaos_get_count(kaos_handle *h, int32_t tube, int64_t *nion, int64_t *nena) {
  if (!h || tube < 0 || tube >= h->ntubes) return KAOS_ERR_PARAM;
  CK(cudaStreamSynchronize(h->s));
  int64_t nl = 0;
  CK(cudaMemcpy(&nl, h->d_nlive + tube, sizeof(int64_t), cudaMemcpyDeviceToHost));
  // slots converted to ENAs or marked at a removal (DEAD) are not ions:
  // the live slots are counted on the device (the export's count and scan)
  int64_t live = 0;
  if (nl) {
    ExportArgs a{};
    a.ion = h->ion[h->cur];
    a.off = h->th[tube].off;
    a.nl = nl;
    a.nb = (int)ceil_div(nl, (int64_t)EXP_THREADS * EXP_ITEMS);
    a.blkoff = (unsigned long long *)h->d_blkoff;
    a.blkcnt = (unsigned *)h->d_blkcnt;
    a.total = (unsigned long long *)(h->d_nlive_new + tube);
    k_exp_count<<<a.nb, EXP_THREADS, 0, h->s>>>(a);
    k_exp_scan<<<1, 1024, 0, h->s>>>(a);
    CK(cudaGetLastError());
    unsigned long long t = 0;
    CK(cudaMemcpyAsync(&t, a.total, sizeof(t), cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    live = (int64_t)t;
  }
  if (nion) *nion = live;
  int64_t ne = 0;
  if (h->d_nena) {
    CK(cudaMemcpy(&ne, h->d_nena + tube, sizeof(int64_t), cudaMemcpyDeviceToHost));
    ne = std::min(ne, h->th[tube].ecap);
  }
  if (nena) *nena = ne;
  return KAOS_OK;
}

int kaos_get_moments(kaos_handle *h, int32_t tube, int32_t which, double *out,
                     int32_t nq) {
  if (!h || !out || tube < 0 || tube >= h->ntubes || which < 0 ||
      which >= KAOS_NMOMENTS)
    return KAOS_ERR_PARAM;
  if (nq != h->th[tube].nq) return fail(h, KAOS_ERR_PARAM, "nq mismatch");
  CK(cudaStreamSynchronize(h->s));
  CK(cudaMemcpy(out, h->ct.mom + which * h->ncell + h->th[tube].coff,
                nq * sizeof(double), cudaMemcpyDeviceToHost));
  return KAOS_OK;
}

int kaos_get_moments_all(kaos_handle *h, int32_t tube, double *out, int32_t nq) {
  if (!h || !out || tube < 0 || tube >= h->ntubes) return KAOS_ERR_PARAM;
  if (nq != h->th[tube].nq) return fail(h, KAOS_ERR_PARAM, "nq mismatch");
  // rows of the [KAOS_NMOMENTS][ncell] block, the tube's nq cells of each
  CK(cudaMemcpy2DAsync(out, (size_t)nq * sizeof(double),
                       h->ct.mom + h->th[tube].coff, (size_t)h->ncell * sizeof(double),
                       (size_t)nq * sizeof(double), KAOS_NMOMENTS,
                       cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  return KAOS_OK;
}

int kaos_get_counts(kaos_handle *h, int32_t tube, int64_t *out, int64_t nbins) {
  if (!h || !out || tube < 0 || tube >= h->ntubes) return KAOS_ERR_PARAM;
  const TubeD &T = h->th[tube];
  CK(cudaStreamSynchronize(h->s));
  if (nbins == T.nq) {
    std::vector<unsigned> v(T.nq);
    CK(cudaMemcpy(v.data(), h->acc.cnt + T.coff, T.nq * sizeof(unsigned), cudaMemcpyDeviceToHost));
    for (int k = 0; k < T.nq; ++k) out[k] = v[k];
    return KAOS_OK;
  }
  if (nbins != (int64_t)T.nq * h->nv) return fail(h, KAOS_ERR_PARAM, "nbins must be nq or nq*nv");
  if (!h->acc.hist) return fail(h, KAOS_ERR_STATE, "full histogram needs kaos_set_export(h, 1)");
  std::vector<unsigned> v(nbins);
  CK(cudaMemcpy(v.data(), h->acc.hist + T.hoff, nbins * sizeof(unsigned), cudaMemcpyDeviceToHost));
  for (int64_t k = 0; k < nbins; ++k) out[k] = v[k];
  return KAOS_OK;
}

int kaos_get_particles(kaos_handle *h, int32_t tube, double *q, double *vpar,
                       double *vperp1, double *vperp2, int32_t *qind,
                       int64_t n) {
  if (!h || tube < 0 || tube >= h->ntubes) return KAOS_ERR_PARAM;
  const TubeD &T = h->th[tube];
  CK(cudaStreamSynchronize(h->s));
  int64_t nl = 0;
  CK(cudaMemcpy(&nl, h->d_nlive + tube, sizeof(int64_t), cudaMemcpyDeviceToHost));
  if (nl == 0) {
    if (n != 0) return fail(h, KAOS_ERR_PARAM, "n (%lld) must equal the ion count (0)", (long long)n);
    return KAOS_OK;
  }
  // the export runs on the device into the spare buffer set (no
  // allocation): q, V||, Vperp1, Vperp2 (FP64) and Qindk1 of the live ions
  // in particle order; the block counts and offsets use the packing's
  // per-block arrays, the total the packing's new-count slot of the tube
  ExportArgs a{};
  a.ion = h->ion[h->cur];
  a.off = T.off;
  a.nl = nl;
  a.qGL = h->ct.qGL + T.coff;
  a.qGH = h->ct.qGH + T.coff;
  a.nq = T.nq;
  a.mixed = h->mixed;
  a.nb = (int)ceil_div(nl, (int64_t)EXP_THREADS * EXP_ITEMS);
  double *dq[4];
  int32_t *dqi = nullptr;
  spare_slots(h, tube, dq, &dqi);
  a.q = q ? dq[0] : nullptr;
  a.vpar = vpar ? dq[1] : nullptr;
  a.v1 = vperp1 ? dq[2] : nullptr;
  a.v2 = vperp2 ? dq[3] : nullptr;
  a.qind = qind ? dqi : nullptr;
  a.blkoff = (unsigned long long *)h->d_blkoff;
  a.blkcnt = (unsigned *)h->d_blkcnt;
  a.total = (unsigned long long *)(h->d_nlive_new + tube);
  k_exp_count<<<a.nb, EXP_THREADS, 0, h->s>>>(a);
  k_exp_scan<<<1, 1024, 0, h->s>>>(a);
  k_exp_write<<<a.nb, EXP_THREADS, 0, h->s>>>(a);
  unsigned long long live = 0;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&live, a.total, sizeof(live), cudaMemcpyDeviceToHost, h->s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->s);
  if (e == cudaSuccess && (int64_t)live != n)
    return fail(h, KAOS_ERR_PARAM, "n (%lld) must equal the ion count (%lld)", (long long)n, (long long)live);
  double *dst[4] = {q, vpar, vperp1, vperp2};
  for (int k = 0; k < 4 && e == cudaSuccess; ++k)
    if (dst[k] && n) e = cudaMemcpyAsync(dst[k], dq[k], n * sizeof(double), cudaMemcpyDeviceToHost, h->s);
  if (e == cudaSuccess && qind && n)
    e = cudaMemcpyAsync(qind, dqi, n * sizeof(int32_t), cudaMemcpyDeviceToHost, h->s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->s);
  if (e != cudaSuccess) return fail(h, KAOS_ERR_CUDA, "get_particles: %s", cudaGetErrorString(e));
  return KAOS_OK;
}

int kaos_get_positions(kaos_handle *h, int32_t tube, double *rho, double *z,
                       int64_t n) {
  if (!h || tube < 0 || tube >= h->ntubes) return KAOS_ERR_PARAM;
  const TubeD &T = h->th[tube];
  CK(cudaStreamSynchronize(h->s));
  int64_t nl = 0;
  CK(cudaMemcpy(&nl, h->d_nlive + tube, sizeof(int64_t), cudaMemcpyDeviceToHost));
  const Ions &I = h->ion[h->cur];
  std::vector<int32_t> qi(nl);
  std::vector<double> a(nl), b(nl);
  if (nl) CK(cudaMemcpy(qi.data(), I.qind + T.off, nl * 4, cudaMemcpyDeviceToHost));
  if (h->mixed) {
    std::vector<double> qv(n);
    int rc = kaos_get_particles(h, tube, qv.data(), nullptr, nullptr, nullptr, nullptr, n);
    if (rc) return rc;
    for (int64_t j = 0; j < n; ++j) {
      double rr = 0.0, zz = 0.0;
      host_rho_z(qv[j], T.pG, &rr, &zz);
      if (rho) rho[j] = rr;
      if (z) z[j] = zz;
    }
    return KAOS_OK;
  }
  if (nl) {
    CK(cudaMemcpy(a.data(), I.rho + T.off, nl * 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(b.data(), I.z + T.off, nl * 8, cudaMemcpyDeviceToHost));
  }
  int64_t k = 0;
  for (int64_t j = 0; j < nl; ++j) {
    if (qi[j] == DEAD) continue;
    if (k >= n) return fail(h, KAOS_ERR_PARAM, "n too small");
    if (rho) rho[k] = a[j];
    if (z) z[k] = b[j];
    ++k;
  }
  return KAOS_OK;
}

int kaos_get_enas(kaos_handle *h, int32_t tube, double *x, double *y, double *z,
                  double *vx, double *vy, double *vz, int64_t n) {
  if (!h || tube < 0 || tube >= h->ntubes) return KAOS_ERR_PARAM;
  int64_t ni = 0, ne = 0;
  int rc = kaos_get_count(h, tube, &ni, &ne);
  if (rc) return rc;
  if (n != ne) return fail(h, KAOS_ERR_PARAM, "n (%lld) must equal the ENA count (%lld)", (long long)n, (long long)ne);
  if (ne == 0) return KAOS_OK;
  const Enas &E = h->ena[h->ecur];
  const int64_t o = h->th[tube].eoff;
  double *dst[6] = {x, y, z, vx, vy, vz};
  double *src[6] = {E.x, E.y, E.z, E.vx, E.vy, E.vz};
  for (int k = 0; k < 6; ++k)
    if (dst[k]) CK(cudaMemcpy(dst[k], src[k] + o, ne * sizeof(double), cudaMemcpyDeviceToHost));
  return KAOS_OK;
}

int kaos_get_boundary(kaos_handle *h, int32_t tube, int64_t *lb_out,
                      int64_t *ub_out, int64_t *lb_in, int64_t *ub_in) {
  if (!h || tube < 0 || tube >= h->ntubes) return KAOS_ERR_PARAM;
  CK(cudaStreamSynchronize(h->s));
  unsigned long long v[4] = {0, 0, 0, 0};
  CK(cudaMemcpy(&v[0], h->d_lb_out + tube, 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(&v[1], h->d_ub_out + tube, 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(&v[2], h->d_lb_in + tube, 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(&v[3], h->d_ub_in + tube, 8, cudaMemcpyDeviceToHost));
  if (lb_out) *lb_out = (int64_t)v[0];
  if (ub_out) *ub_out = (int64_t)v[1];
  if (lb_in) *lb_in = (int64_t)v[2];
  if (ub_in) *ub_in = (int64_t)v[3];
  return KAOS_OK;
}

int kaos_get_boundary_ena(kaos_handle *h, int32_t tube, int64_t *lb_out,
                          int64_t *ub_out) {
  if (!h || tube < 0 || tube >= h->ntubes) return KAOS_ERR_PARAM;
  unsigned long long v[2] = {0, 0};
  if (h->d_lbe_out) {
    CK(cudaStreamSynchronize(h->s));
    CK(cudaMemcpy(&v[0], h->d_lbe_out + tube, 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&v[1], h->d_ube_out + tube, 8, cudaMemcpyDeviceToHost));
  }
  if (lb_out) *lb_out = (int64_t)v[0];
  if (ub_out) *ub_out = (int64_t)v[1];
  return KAOS_OK;
}

int kaos_get_timing(kaos_handle *h, double *ms, int64_t *launches) {
  if (!h) return KAOS_ERR_PARAM;
  if (ms) *ms = h->last_ms;
  if (launches) *launches = h->launches;
  return KAOS_OK;
}

int kaos_get_push_timing(kaos_handle *h, double *ms, int64_t *launches) {
  if (!h) return KAOS_ERR_PARAM;
  if (ms) *ms = h->push_ms;
  if (launches) *launches = h->npev;
  return KAOS_OK;
}

int kaos_sample_rng(int32_t kind, uint64_t seed, uint64_t id0, uint32_t step,
                    uint32_t c3, double lambda, int64_t n, double *out) {
  if (kind < KAOS_SAMPLE_PHILOX || kind > KAOS_SAMPLE_GAUSS64T || n < 0 ||
      n > ((int64_t)1 << 26) || (n > 0 && !out) ||
      (kind == KAOS_SAMPLE_POISSON && !(lambda >= 0.0 && lambda <= 700.0)))
    return KAOS_ERR_PARAM;
  if (n == 0) return KAOS_OK;
  const int per = sample_width(kind);
  double *d = nullptr;
  if (cudaMalloc(&d, (size_t)n * per * sizeof(double)) != cudaSuccess) return KAOS_ERR_CUDA;
  SampleArgs a{};
  a.kind = kind;
  a.seed = seed;
  a.id0 = id0;
  a.step = step;
  a.c3 = c3;
  a.lambda = lambda;
  a.n = n;
  a.out = d;
  for (int r = 0; r < 10; ++r) {  // Philox key schedule of the seed
    a.rk[2 * r] = (uint32_t)seed + (uint32_t)r * KAOS_PHILOX_W0;
    a.rk[2 * r + 1] = (uint32_t)(seed >> 32) + (uint32_t)r * KAOS_PHILOX_W1;
  }
  k_sample_rng<<<(int)std::min<int64_t>((n + 255) / 256, 148 * 16), 256>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpy(out, d, (size_t)n * per * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(d);
  return e == cudaSuccess ? KAOS_OK : KAOS_ERR_CUDA;
}

void kaos_destroy(kaos_handle *h) {
  if (!h) return;
  if (g_grid_owner == h) g_grid_owner = nullptr;
  if (h->s) cudaStreamSynchronize(h->s);
  if (h->s2) cudaStreamSynchronize(h->s2);
  for (auto &g : h->graphs) cudaGraphExecDestroy(g.second.exec);
  for (auto e : h->pev) cudaEventDestroy(e);
  for (void *p : h->allocs) cudaFree(p);
  if (h->e0) cudaEventDestroy(h->e0);
  if (h->e1) cudaEventDestroy(h->e1);
  if (h->conv_host.stage) cudaFreeHost(h->conv_host.stage);
  if (h->cx_stat) cudaFreeHost(h->cx_stat);
  if (h->efork) cudaEventDestroy(h->efork);
  if (h->ejoin) cudaEventDestroy(h->ejoin);
  if (h->s2) cudaStreamDestroy(h->s2);
  if (h->s) cudaStreamDestroy(h->s);
  delete h;
}

}  // extern "C"

// ===========================================================================
// Allocation-free statistics entry point (kaos_moments_noalloc).
//
// Some callers cannot call cudaMalloc: a Fortran or C host that runs under a
// fixed device-memory budget handed out by its own pool, and processes that
// share a GPU under an externally enforced memory cap.  For them the
// start-of-step statistics -- per-cell counts and the moment integrals of
// IonParticleCountsSub and the ZerothIonMoment .. SecondParIonMoment
// routines -- run here with every intermediate histogram in one file-scope
// device array instead of allocated scratch.  The caller passes the
// particle inputs and the outputs; this code allocates nothing.  The
// velocity grid travels by value in the kernel arguments (no host-to-device
// copy of a host buffer).
//
// The array holds NOALLOC_MAX_CELLS cells x (1 + 3 * MAXV) 32-bit counters
// (about 0.79 MB) and lives in every GPU that loads the library until the
// process exits.  Its contents persist between calls: each call clears the
// part it uses before binning.  All calls share the one array, so calls
// that overlap on the GPU (two streams, two host threads) race; serialise
// them.
namespace {

constexpr int NOALLOC_MAX_CELLS = 512;
constexpr size_t NOALLOC_WORDS = (size_t)NOALLOC_MAX_CELLS * (1 + 3 * MAXV);

static __device__ __align__(256) unsigned int g_noalloc_scratch[NOALLOC_WORDS];

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mutex;
unsigned int *g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {nullptr};
int g_noalloc_nsm[NOALLOC_MAX_DEVICES] = {0};

// The three axes' FP64 edges of the by-value grid, copied into shared
// memory (searched there by every thread).
__device__ __forceinline__ void noalloc_edges(const VGridC &vg, double *s1,
                                              double *s2, double *sp) {
  for (int k = threadIdx.x; k <= MAXV; k += blockDim.x) {
    s1[k] = vg.e1[k];
    s2[k] = vg.e2[k];
    sp[k] = vg.epar[k];
  }
}

// per-particle cell / velocity-bin search and counting into the scratch
__global__ void k_noalloc_bin(unsigned *scr, const VGridC vg, const double *qedges,
                              int nq, const double *q, const double *vpar,
                              const double *v1, const double *v2, int64_t n) {
  extern __shared__ double E[];
  __shared__ double S1[MAXV + 1], S2[MAXV + 1], SP[MAXV + 1];
  // orientation: q increases upward when the lower boundary has q <= 0
  const double sgn = qedges[0] <= 0.0 ? 1.0 : -1.0;
  for (int k = threadIdx.x; k <= nq; k += blockDim.x) E[k] = sgn * qedges[k];
  noalloc_edges(vg, S1, S2, SP);
  __syncthreads();
  const int n1 = vg.n1, n2 = vg.n2, npar = vg.npar, d3 = vg.three_d;
  unsigned *cnt = scr, *mpar = scr + NOALLOC_MAX_CELLS,
           *m1 = mpar + (size_t)NOALLOC_MAX_CELLS * MAXV,
           *m2 = m1 + (size_t)NOALLOC_MAX_CELLS * MAXV;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x) {
    const int c = cell_search(E, nq, sgn * q[j]);
    if (c < 0) continue;
    atomicAdd(cnt + c, 1u);
    const double a = v1[j], b = v2 ? v2[j] : 0.0;
    const int bp = vbin(SP, npar, vpar[j]);
    const int b1 = vbin(S1, n1, d3 ? a : vperp_mag(a, b));
    const int b2 = d3 ? vbin(S2, n2, b) : 0;
    if (bp < 0 || b1 < 0 || b2 < 0) continue;
    atomicAdd(mpar + (size_t)c * MAXV + bp, 1u);
    atomicAdd(m1 + (size_t)c * MAXV + b1, 1u);
    if (d3) atomicAdd(m2 + (size_t)c * MAXV + b2, 1u);
  }
}

__global__ void k_noalloc_moments(const unsigned *scr, const VGridC vg, int nq,
                                  const double *d3x, double nsnormfac, double ms,
                                  int cenpar, int cenperp, double *out,
                                  int64_t *counts) {
  __shared__ double S1[MAXV + 1], S2[MAXV + 1], SP[MAXV + 1];
  noalloc_edges(vg, S1, S2, SP);
  __syncthreads();
  const unsigned *cnt = scr, *mpar = scr + NOALLOC_MAX_CELLS,
                 *m1 = mpar + (size_t)NOALLOC_MAX_CELLS * MAXV,
                 *m2 = m1 + (size_t)NOALLOC_MAX_CELLS * MAXV;
  for (int Q = threadIdx.x; Q < nq; Q += blockDim.x) {
    const double w = nsnormfac / d3x[Q];
    double M[10];
    cell_moments(w, (double)cnt[Q], mpar + (size_t)Q * MAXV, m1 + (size_t)Q * MAXV,
                 m2 + (size_t)Q * MAXV, SP, S1, S2, vg.npar, vg.n1, vg.n2,
                 vg.three_d, cenpar, cenperp, ms, M);
    for (int k = 0; k < 10; ++k) out[(size_t)k * nq + Q] = M[k];
    out[(size_t)KAOS_NQ * nq + Q] = (double)cnt[Q] * w;
    if (counts) counts[Q] = cnt[Q];
  }
}

}  // namespace

extern "C" int kaos_moments_noalloc(const kaos_params_c *p,
                                    const kaos_vgrid_c *vgc, int32_t nq,
                                    const double *d_qedges, const double *d_d3x,
                                    double nsnormfac, const double *d_q,
                                    const double *d_vpar, const double *d_vperp1,
                                    const double *d_vperp2, int64_t n,
                                    double *d_moments, int64_t *d_counts,
                                    void *stream) {
  if (!p || !vgc || !d_qedges || !d_d3x || !d_moments || n < 0 ||
      (n > 0 && (!d_q || !d_vpar || !d_vperp1)))
    return KAOS_ERR_PARAM;
  const int d3 = p->ION2VPERPflag == 1;
  // a 3D grid bins Vperp2 on its own axis: the array is required
  if (d3 && n > 0 && !d_vperp2) return KAOS_ERR_PARAM;
  if (nq < 1 || nq > NOALLOC_MAX_CELLS) return KAOS_ERR_CAPACITY;
  if (vgc->n1 < 1 || vgc->n1 > MAXV || vgc->npar < 1 || vgc->npar > MAXV ||
      (d3 && (vgc->n2 < 1 || vgc->n2 > MAXV || !vgc->e2)) || !vgc->e1 || !vgc->epar)
    return KAOS_ERR_CAPACITY;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES)
    return KAOS_ERR_CUDA;
  // set-up once per device, with that device current: host code needs the
  // device address of the array (its name here is only a host stand-in),
  // and the grid of the binning kernel is sized by the device's SM count
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
      void *a = nullptr;
      int nsm = 0;
      if (cudaGetSymbolAddress(&a, g_noalloc_scratch) != cudaSuccess) return KAOS_ERR_CUDA;
      if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
          nsm < 1)
        return KAOS_ERR_CUDA;
      g_noalloc_nsm[dev] = nsm;
      g_noalloc_ptr[dev] = (unsigned *)a;
    }
  }
  unsigned *scr = g_noalloc_ptr[dev];
  cudaStream_t s = (cudaStream_t)stream;
  VGridC vg{};
  vg.three_d = d3;
  vg.n1 = vgc->n1;
  vg.n2 = d3 ? vgc->n2 : 0;
  vg.npar = vgc->npar;
  for (int k = 0; k <= vg.n1; ++k) vg.e1[k] = vgc->e1[k];
  for (int k = 0; k <= vg.npar; ++k) vg.epar[k] = vgc->epar[k];
  for (int k = 0; d3 && k <= vg.n2; ++k) vg.e2[k] = vgc->e2[k];
  if (cudaMemsetAsync(scr, 0, NOALLOC_WORDS * sizeof(unsigned), s) != cudaSuccess)
    return KAOS_ERR_CUDA;
  if (n > 0) {
    // 8 blocks of 256 threads per SM stride over the ions
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)g_noalloc_nsm[dev] * 8);
    k_noalloc_bin<<<blocks, 256, (size_t)(nq + 1) * sizeof(double), s>>>(
        scr, vg, d_qedges, nq, d_q, d_vpar, d_vperp1, d_vperp2, n);
  }
  k_noalloc_moments<<<1, 256, 0, s>>>(scr, vg, nq, d_d3x, nsnormfac, p->ms,
                                      p->PHASEENERGYPARIONMOMENTCENTERflag == 1,
                                      p->PHASEENERGYPERPIONMOMENTCENTERflag == 1,
                                      d_moments, d_counts);
  if (cudaGetLastError() != cudaSuccess) return KAOS_ERR_CUDA;
  return KAOS_OK;
}
