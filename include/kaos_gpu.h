/*
 * kaos_gpu.h -- C-ABI of the B200 kinetic particle loop for KAOS
 * (Kinetic model of Auroral ion OutflowS).
 *
 * The reference has no plugin API: its hot path is the body of
 * `KineticSolverSub` (_8_KineticSolver.f90:35-263), reached by the single
 * call `call KineticSolverSub` (_KineticMain.f90:41), with all state held
 * in module globals (_KineticMainParams.f90:170-250).  Each entry point
 * below replaces one block of that body; the comment on each names the
 * reference lines it stands for.  A Fortran host binds these through the
 * `bind(C)` interface in kaos_b200/fortran/kaos_gpu_iface.f90.
 *
 * Conventions
 *  - SI units throughout, like the reference.
 *  - Configuration cells are 0-based inside the library (reference Qind =
 *    NqLB + k).  Exported cell indices keep the reference escape sentinels
 *    shifted to negative values: -1 = below the lower boundary (reference
 *    Qind 0), -2 = above the upper boundary (reference Qind -1).
 *  - Velocity-bin indices are 0-based; -1 = outside the velocity grid
 *    (reference index 0).
 *  - Every call returns an int status (KAOS_OK on success).  The text of
 *    the last error of a handle is returned by kaos_last_error().
 *  - A handle owns one CUDA stream on the device that was current when it
 *    was created and is not thread safe; use one handle per thread/GPU.
 */
#ifndef KAOS_GPU_H
#define KAOS_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define KAOS_OK 0
#define KAOS_ERR_PARAM 1    /* bad argument / inconsistent parameters      */
#define KAOS_ERR_CAPACITY 2 /* particle capacity of a tube exceeded        */
#define KAOS_ERR_NAN 3      /* non-finite particle state detected          */
#define KAOS_ERR_CUDA 4     /* CUDA runtime error                          */
#define KAOS_ERR_TIMEOUT 5  /* reserved: no kernel here waits on another, */
                            /* so this build never returns it             */
#define KAOS_ERR_STATE 6    /* call out of order (e.g. step before load)   */

/* ---- precision modes ---------------------------------------------------- */
#define KAOS_PREC_FP64 0  /* all particle arithmetic in FP64                */
#define KAOS_PREC_MIXED 1 /* FP32 forces, RK stages and heating kicks on
                             FP64 state (position, V||, Vperp); FP64 quartic,
                             renormalisation and reductions                  */
#define KAOS_PREC_MIXED_K64 2 /* KAOS_PREC_MIXED with the WaveHeatingSub kick
                             (_8_1_1_0_WaveHeating.f90:72-312) in FP64: the
                             FP64 path's formula and random draw on the FP64
                             state, so heated runs keep the FP64 path's bins */

/* ---- moment selectors for kaos_get_moments ------------------------------ */
#define KAOS_M0 0        /* M0phRT      density [m^-3]                      */
#define KAOS_M1PERP1 1   /* M1Perp1phRT [m/s]   (3D velocity grid)          */
#define KAOS_M1PERP2 2   /* M1Perp2phRT [m/s]   (3D velocity grid)          */
#define KAOS_M1PAR 3     /* M1ParphRT   [m/s]                               */
#define KAOS_M2 4        /* M2phRT      [J]                                 */
#define KAOS_M2PERP1 5   /* M2Perp1phRT [J]     (3D velocity grid)          */
#define KAOS_M2PERP2 6   /* M2Perp2phRT [J]     (3D velocity grid)          */
#define KAOS_M2PAR 7     /* M2ParphRT   [J]                                 */
#define KAOS_M1PERP 8    /* M1PerpphRT  [m/s]   (2D velocity grid)          */
#define KAOS_M2PERP 9    /* M2PerpphRT  [J]     (2D velocity grid)          */
#define KAOS_NQ 10       /* NqRT  per-cell density from counts [m^-3]       */
#define KAOS_EAMAG 11    /* EAmagRT ambipolar field at cell centres [V/m]   */
#define KAOS_EGMAG 12    /* EGmagRT gravity "field" at cell centres [V/m]   */
#define KAOS_M0FILT 13   /* M0FiltAvrgRT filtered density used by EAmag     */
#define KAOS_NUPOI 14    /* nuIonNeutRT Poisson collision counts per cell  */
/* ENA statistics (charge exchange on), on the ENA velocity grid (Vp, Vq,
 * Vphi) of kaos_set_ena_grid: ENAParticleCountsSub
 * (_8_3_2_ENAParticleCounts.f90) and ZerothENAMoment .. SecondPHIENAMoment
 * (_8_10_1 .. _8_10_8). */
#define KAOS_ENA_NQ 15     /* NqENART  ENA density from counts [m^-3]      */
#define KAOS_ENA_M0 16     /* M0phENART    [m^-3]                          */
#define KAOS_ENA_M1P 17    /* M1PphENART   [m/s]                           */
#define KAOS_ENA_M1Q 18    /* M1QphENART   [m/s]                           */
#define KAOS_ENA_M1PHI 19  /* M1PHIphENART [m/s]                           */
#define KAOS_ENA_M2 20     /* M2phENART    [eV]                            */
#define KAOS_ENA_M2P 21    /* M2PphENART   [eV]                            */
#define KAOS_ENA_M2Q 22    /* M2QphENART   [eV]                            */
#define KAOS_ENA_M2PHI 23  /* M2PHIphENART [eV]                            */
#define KAOS_NMOMENTS 24

/*
 * Run parameters: the subset of _ModelInput.f90 / FluxTubeT flag fields
 * (_KineticMainParams.f90:464-473) that the per-step loop reads.  Flags are
 * 0/1 exactly as in the reference.
 */
typedef struct kaos_params_c {
  double ms;       /* SpecieT%msT ion mass [kg]                        */
  double qs;       /* SpecieT%qsT ion charge [C]                       */
  double h;        /* SpecieT%hT computational time step [s]           */
  double mNeut;    /* neutral mass for ENA gravity / collisions [kg]   */
  double TNeut;    /* neutral temperature [K]                          */
  double dNTe;     /* Te increment per master step [K]                 */
  double dNTeEND;  /* Te increment cap [K]                             */
  uint64_t seed;   /* counter-based RNG key                            */
  int32_t ndatfac; /* master-step cadence (reference ndatfacGT)        */
  int32_t precision;            /* KAOS_PREC_*                         */
  int32_t ION2VPERPflag;        /* 1: 3D (Vperp1,Vperp2,Vpar) grid     */
  int32_t ICRflag;              /* wave heating                        */
  int32_t ICRCOHERENCEflag;     /* coherent heating variant            */
  int32_t MIRRORflag;
  int32_t GRAVflag;
  int32_t EAMBflag;
  int32_t EAMBSIGNflag;
  int32_t EAMBSELFCONSISTflag;
  int32_t EAPRESSUREflag;
  int32_t MOMENTFILTERflag;
  int32_t QEXCHANGEflag;        /* ion -> ENA charge exchange          */
  int32_t LBCONDITIONflag;      /* lower-boundary injection            */
  int32_t UBCONDITIONflag;      /* upper-boundary injection            */
  int32_t STATICINJECTIONflag;
  int32_t PHASEENERGYPARIONMOMENTCENTERflag;
  int32_t PHASEENERGYPERPIONMOMENTCENTERflag;
  int32_t M0MAfilterPt;         /* moving-average points (odd)         */
  int32_t M1ParMAfilterPt;
  int32_t M1Perp1MAfilterPt;
  int32_t M1Perp2MAfilterPt;
  int32_t M2ParMAfilterPt;
  int32_t FLUXINJECTIONflag;  /* 1: injected V|| drawn from the Maxwellian
                                 flux through the boundary (directed into the
                                 tube) instead of the plain Maxwellian of
                                 _8_0_0_2_KineticSolverB.f90:317-335; an
                                 extension, 0 in the reference's runs      */
  int32_t reserved[3];
} kaos_params_c;

/*
 * One flux tube: the per-cell grid tables of FluxTubeT
 * (_KineticMainParams.f90:476-481) for the cells NqLB..NqUB, flattened to
 * 0-based arrays of length nq.  All pointers are host pointers read once by
 * kaos_create.  Optional tables may be NULL (zeros are used).
 */
typedef struct kaos_tube_c {
  int32_t nq;              /* NqUB - NqLB + 1, in [6, 2048]                */
  int32_t capacity;        /* max particles (incl. injection headroom)     */
  double pG;               /* pGCGT  (field-line p = L shell) [RE]         */
  double phiG;             /* phiGCGT longitude [rad]                      */
  double nsnormfac;        /* macro-particle weight                        */
  double nsnormCLB;        /* LB injection macro-particle count / master   */
  double nsnormCUB;        /* UB injection macro-particle count / master   */
  double sumdsICR;         /* sum(dsICRGT) heating-region arc length [m]   */
  const double *qGL, *qGH, *qGC;   /* cell lower/upper/centre q            */
  const double *hqC, *dqC, *d3xC;  /* metric factor, width, volume         */
  const double *rGC, *thetaGC, *ellGC; /* cell-centre r, theta, ell        */
  const double *TeG;       /* TeGT electron temperature [K]                */
  const double *TsG;       /* TsGT ion temperature (injection) [K]         */
  const double *nsnormCNeut; /* neutral density for collisions [m^-3]      */
  /* ICR wave-heating tables (_1_SimParameterization.f90:1408-1444)        */
  const double *lambdaPerp, *EtaLH, *XiPerp1, *XiPerp2;
  const double *S0, *OmegaG0, *ChiPerp1, *ChiPerp2;
  /* species of this entry (SpecieT(s)%msT, qsT); 0 = kaos_params_c ms/qs.
   * Several species of one flux tube are separate entries: the reference
   * runs species as independent outermost loops (_8_KineticSolver.f90:43),
   * each with the ambipolar field of its own density. */
  double ms, qs;
} kaos_tube_c;

/*
 * The velocity grid, shared by every cell and tube (the reference reads
 * QCellT(1)%V2PerpCellT everywhere, e.g. _8_4_1_IonDistributionFunctions
 * .f90:58-59).  Edges are separable per axis.
 *   3D (ION2VPERPflag=1): axes Vperp1 (n1), Vperp2 (n2), Vpar (npar).
 *   2D (ION2VPERPflag=0): axes Vperp (n1, magnitudes), Vpar (npar); n2=0.
 * Arrays of edges have n+1 entries (lower edge of bin k = e[k], upper =
 * e[k+1]); centres are (lo+hi)/2 as in _0_0_VelGridGenerator.f90:338-467.
 */
typedef struct kaos_vgrid_c {
  int32_t n1, n2, npar;
  const double *e1, *e2, *epar;
} kaos_vgrid_c;

typedef struct kaos_handle kaos_handle;

/* Create a solver for `ntubes` independent tubes on the current device.
 * Replaces the allocation and parameter copy of DataTypeAllocBSub /
 * SimParameterizationSub (_8_KineticSolver.f90:50).  With
 * MOMENTFILTERflag = 1 every moving-average window must be odd, >= 3 and at
 * most the tube's cell count (MomentFilterSub reads that many cells around
 * each cell; the reference's guard, NqICT >= (Pt-1)/2, lets shorter tubes
 * read outside the array).  With QEXCHANGEflag = 1 at most KAOS_MAX_TUBES_CX
 * tubes (the ENA push holds a per-tube prefix in shared memory); more
 * return KAOS_ERR_PARAM. */
#define KAOS_MAX_TUBES_CX 32768
int kaos_create(const kaos_params_c *p, const kaos_tube_c *tubes,
                int32_t ntubes, const kaos_vgrid_c *vg, kaos_handle **out);

/* Load the initial particles of one tube: the initial-condition arrays
 * x0T..Vz0T, Vperp10T, Vperp20T of FluxTubeT (_7_InitialConditions.f90:
 * 51-98).  Positions are field-line q values (p = pG is implied);
 * velocities are field-aligned components.  The arrays are staged through
 * the library's spare particle buffers (no device allocation); pinned host
 * arrays copy fastest. */
int kaos_load_particles(kaos_handle *h, int32_t tube, const double *q,
                        const double *vpar, const double *vperp1,
                        const double *vperp2, int64_t n);

/*
 * Initial ions generated on the device, in place of kaos_load_particles:
 * the steps either side of the loop that DensityProfileA1/B, the velocity
 * distribution and InitialConditions do on the host in the reference
 * (_2_1_DensityProfileA1.f90, _4_DensityProfileB.f90,
 * _6_VelocityDistribution.f90, _7_InitialConditions.f90).  counts[k] ions
 * start in cell k at q uniform over the middle 96 % of the cell; each ion's
 * velocity (V||, Vperp1, Vperp2) is an isotropic Maxwellian at the cell's
 * TsG, or, with probability tail_fraction, an isotropic kappa distribution
 * f ~ (1 + v^2/(kappa theta^2))^-(kappa+1) of temperature tail_T (drawn as
 * a Student-t vector of 2 kappa - 1 degrees of freedom; 2 kappa - 1 must be
 * an integer in [3, 63]).  Random numbers: Philox keyed by (seed, ion index,
 * KAOS_RNG_INIT), the same generator as the CPU oracle's, so both start from
 * the same ions.  Ions are numbered 0..n-1 in cell order.
 */
typedef struct kaos_init_c {
  const int64_t *counts;   /* ions per cell [nq]                           */
  double tail_fraction;    /* fraction of ions from the kappa tail, [0, 1] */
  double kappa;            /* kappa index of the tail                      */
  double tail_T;           /* tail temperature [K]                         */
  uint64_t seed;
} kaos_init_c;

int kaos_init_particles(kaos_handle *h, int32_t tube, const kaos_init_c *init);

/* Set the per-cell ambipolar field EAmagRT (host-imported spin-up
 * profile, _8_7_AmbipolarEfield.f90:1375-1402) used on the first step.
 * NULL resets to "compute from the initial moments". */
int kaos_set_fields(kaos_handle *h, int32_t tube, const double *EAmag,
                    int32_t nq);

/* Advance every tube by `nsteps` computational steps: the body of the
 * ComputationalTimeStepLoop (_8_KineticSolver.f90:54-239): charge exchange,
 * BoundaryConditionsSub, AmbipolarEfieldSub/GravfieldSub, KineticSolverA/B
 * (push, injection, counts, distribution functions, moments).  The first
 * call performs the n=1 step of KineticSolverASub. */
int kaos_step(kaos_handle *h, int64_t nsteps);

/* Number of computational steps taken so far (reference n - 1). */
int kaos_get_step(kaos_handle *h, int64_t *n);

/* Live particle counts of a tube: ions and ENAs (reference NsT split by
 * ENAflag). */
int kaos_get_count(kaos_handle *h, int32_t tube, int64_t *nion,
                   int64_t *nena);

/* Per-cell moment / field of the latest master step (M*phRT(nn,:),
 * EAmagRT(nn,:) ...), `which` = KAOS_M0 ... ; out has nq doubles. */
int kaos_get_moments(kaos_handle *h, int32_t tube, int32_t which,
                     double *out, int32_t nq);

/* Every selector of kaos_get_moments at once, in one device-to-host copy:
 * out[m * nq + k] = selector m (KAOS_M0 ... KAOS_ENA_M2PHI), cell k;
 * out has KAOS_NMOMENTS * nq doubles.  The set DataExport2Sub writes per
 * master step (_8_0_2_DataExport2.f90:29-150) without one call and one
 * synchronisation per moment. */
int kaos_get_moments_all(kaos_handle *h, int32_t tube, double *out, int32_t nq);

/* Integer counts of the latest master step: per-cell ion counts
 * (NqReNormT, nq entries) when nbins == nq, or the full phase-space
 * histogram N2PerpphReNormRT / NphReNormRT laid out
 * [cell][v1][v2][vpar] (3D) or [cell][vperp][vpar] (2D) when nbins equals
 * that size.  The full histogram requires kaos_set_export(h, 1) before the
 * master step. */
int kaos_get_counts(kaos_handle *h, int32_t tube, int64_t *out,
                    int64_t nbins);

/* Enable (1) / disable (0) materialising the full phase-space histogram on
 * master steps (the DataExport2 path). */
int kaos_set_export(kaos_handle *h, int32_t on);

/* Copy the ion state of a tube to host arrays of length n (n must equal the
 * live ion count): field-line q, parallel velocity, Vperp1, Vperp2 and the
 * start-of-step cell index Qindk1 (0-based, -1/-2 escape sentinels).  In
 * mixed precision Qindk1 is stored only by the pushes whose successor reads
 * it (the step before a master step, every step of an interval whose charge
 * exchange converts ions, or every step with export on): elsewhere it is
 * that of the last such step.  Any
 * pointer may be NULL.  Order is the reference particle order.  The state
 * is gathered on the device into the spare particle buffers (no device
 * allocation) and copied once per array. */
int kaos_get_particles(kaos_handle *h, int32_t tube, double *q, double *vpar,
                       double *vperp1, double *vperp2, int32_t *qind,
                       int64_t n);

/* Meridian-plane position (rho = x cos phi + y sin phi, z) of the ions of a
 * tube, FP64 reconstruction of xN/yN/zN (_8_1_KineticRK4Update.f90:174-176). */
int kaos_get_positions(kaos_handle *h, int32_t tube, double *rho, double *z,
                       int64_t n);

/* ENA state of a tube (Cartesian x, y, z, Vx, Vy, Vz), n = live ENA count. */
int kaos_get_enas(kaos_handle *h, int32_t tube, double *x, double *y,
                  double *z, double *vx, double *vy, double *vz, int64_t n);

/* Boundary fluxes of the latest master step: escaped LB/UB ion counts
 * (NqReNormLB/UBoutfluxIonT) and injected LB/UB counts (LB/UBNetDensityT). */
int kaos_get_boundary(kaos_handle *h, int32_t tube, int64_t *lb_out,
                      int64_t *ub_out, int64_t *lb_in, int64_t *ub_in);

/* ENAs that left the tube at the latest master step through the lower and
 * the upper boundary (Qindk1 = 0 / -1; NqReNormLB/UBoutfluxENAT,
 * _8_0_7_BoundaryConditions.f90:305-416).  Zero without charge exchange. */
int kaos_get_boundary_ena(kaos_handle *h, int32_t tube, int64_t *lb_out,
                          int64_t *ub_out);

/* Device time (ms) of the last kaos_step call, measured with CUDA events on
 * the handle's stream, and the number of kernels it launched. */
int kaos_get_timing(kaos_handle *h, double *ms, int64_t *launches);

/* Device time (ms) spent in the particle push kernels alone during the last
 * kaos_step call (CUDA events around each push launch) and their count.
 * Steps replayed from CUDA graphs carry no per-push events and are not
 * included. */
int kaos_get_push_timing(kaos_handle *h, double *ms, int64_t *launches);

/* Diagnostic sampler of the library's device random-number generators, for
 * distribution tests; no counterpart in the reference (whose generators,
 * gfortran's unseeded random_number behind GaussianRNGSub and
 * PoissonRNGSub, _3_1_GaussianRNG.f90:27-37 and _3_2_PoissonRNG.f90:27-42,
 * are not reproducible).  Draw i (i = 0 .. n-1) is evaluated on the device
 * by the same function the kernels call and written to the host array out:
 *   KAOS_SAMPLE_PHILOX  4 values: the Philox4x32-10 words of counter
 *                       (id0 + i low, high, step, c3) and key `seed`;
 *   KAOS_SAMPLE_GAUSS32 2 values: the FP32 Gaussian pair of the mixed
 *                       push's heating kick for particle id0 + i at step;
 *   KAOS_SAMPLE_GAUSS64 2 values: the FP64 Gaussian pair of the FP64 push's
 *                       heating kick for particle id0 + i at step;
 *   KAOS_SAMPLE_POISSON 1 value: the collision-count draw with mean
 *                       `lambda` for cell id0 + i at master step `step`;
 *   KAOS_SAMPLE_GAUSS64T 2 values: the same pair as KAOS_SAMPLE_GAUSS64 as
 *                       the KAOS_PREC_MIXED_K64 push evaluates it (table-
 *                       reduced FP64 logarithm and sine/cosine).
 * out holds 4, 2, 2, 1 or 2 doubles per draw; n <= 2^26. */
#define KAOS_SAMPLE_PHILOX 0
#define KAOS_SAMPLE_GAUSS32 1
#define KAOS_SAMPLE_GAUSS64 2
#define KAOS_SAMPLE_POISSON 3
#define KAOS_SAMPLE_GAUSS64T 4
int kaos_sample_rng(int32_t kind, uint64_t seed, uint64_t id0, uint32_t step,
                    uint32_t c3, double lambda, int64_t n, double *out);

/* Run the computational steps from CUDA graphs (1) or launch every kernel
 * directly (0, default).  With graphs on, each kind of step (ordinary runs
 * of up to 8 steps, the step before a master step, the master step) is
 * captured once per ion/ENA buffer parity and replayed; the step number
 * lives in device memory, so a replay needs no host update.  Results are
 * identical to the direct launches.  Step 1 always runs directly.  No
 * reference counterpart (the Fortran loop calls each routine per step,
 * _8_KineticSolver.f90:54-239). */
int kaos_set_graph(kaos_handle *h, int32_t on);

/* Launch shape of the particle push: `chunk` ions per work item (1024,
 * 2048 or 4096; an item is a (tube, chunk of ions) pair) and `mode` bit 0:
 * 0 = one thread block per item, 1 = a persistent grid (resident blocks per
 * SM x SMs) striding over the items; bits 1-2 (mixed precision only):
 * register budget of the push, 0 = 64 registers (4 blocks of 256 threads
 * per SM), 1 = 80 registers (3 blocks of 256), 2 = 72 registers (7 blocks
 * of 128); bits 3-4 (mixed): the budget of the master-step variant plus
 * one (0 = the same as bits 1-2).  chunk = 0 or mode < 0 re-arms the
 * autotuner, which is on by default: before the first step after step 1 it
 * times the push of every candidate on a copy of the ion state and keeps
 * the fastest, then the master-step variant's budget alone.  Results do not depend on the shape.  No reference
 * counterpart (the reference has one MPI rank per core,
 * _8_KineticSolver.f90:43-44). */
int kaos_set_launch(kaos_handle *h, int32_t chunk, int32_t mode);

/* ENA velocity grid V3CellT (_KineticMainParams.f90:364-399): Vp edges
 * e1[n1+1], Vphi edges e2[n2+1], Vq (= V||) edges epar[npar+1].  Set before
 * the first step; without it the ion grid's axes are used (Vp <- Vperp1,
 * Vq <- Vpar, Vphi <- Vperp2, or Vperp1 on a 2D ion grid). */
int kaos_set_ena_grid(kaos_handle *h, const kaos_vgrid_c *vg);

/*
 * One tube split across ranks (MPI ranks of the reference, one GPU each
 * here): each rank holds a handle with the tube's full tables and its own
 * share of the ions.  The reference sums every per-cell and per-bin count
 * over the ranks (MPIReduceSumSub _9_MPIReduceSum.f90:25-55, called per bin
 * from _8_3_1_IonParticleCounts.f90:396-407, :675-680) before the moments;
 * here the handle calls `fn(ctx, buf, count, stream)` once per statistics
 * step with ALL its binning accumulators in one device block of `count`
 * uint32 counters (ion and ENA counts and marginals), after synchronising
 * its stream.  The hook sums `buf` over the ranks in place (an NCCL
 * all-reduce, kaos_b200/shard.py) and returns 0 when done.  While a hook is
 * set, steps run without CUDA graphs.  fn = NULL removes it.
 */
typedef int (*kaos_reduce_fn)(void *ctx, uint32_t *buf, int64_t count,
                              void *stream);
int kaos_set_reduce(kaos_handle *h, kaos_reduce_fn fn, void *ctx);

/* Rank `rank` of `nranks` holding a share of a split tube: of the
 * nint(nuIonNeutPoiT) ions a cell converts to ENAs at a step (IonNeutral
 * CollisionFrequencyBSub splits the count over ranks,
 * _8_6_6_2_IonNeutralCollisionFrequencyB.f90), this rank converts
 * floor((N + rank) / nranks), its first ones in index order. */
int kaos_set_rank(kaos_handle *h, int32_t rank, int32_t nranks);

/* Id of the first ion loaded into `tube` (default 0): ids key the random
 * streams of each ion, so the shares of a split tube take disjoint ranges
 * and draw the same numbers as the unsplit tube.  Set before loading. */
int kaos_set_id_base(kaos_handle *h, int32_t tube, uint64_t base);

/*
 * Convection of a tube to a new L-shell (ConvectionSub, _8_11_Convection
 * .f90:135-258; the reference's E x B L-shell update is a stub adding 0,
 * :107, and its grid keeps the q boundaries qGA/qGB).  `t` holds the tube's
 * tables regenerated for the new pG (and phiG) on the same q grid (same nq,
 * qGL, qGH).  At the next master step, before anything else, every ion keeps
 * its q and V|| and moves to the new field line, its magnetic moment kept:
 * both Vperp components scale by sqrt(B_new/B_old); then the new tables
 * replace the old.  ENAs are neutral and stay where they are.  The tube's
 * evolving Te is kept.
 */
int kaos_update_tube(kaos_handle *h, int32_t tube, const kaos_tube_c *t);

/* The launch shape in use (after autotuning); mode bits 3-4 are 0 when
 * the master-step variant uses the same register budget as the push. */
int kaos_get_launch(kaos_handle *h, int32_t *chunk, int32_t *mode);

/* Text of the last error on this handle (static storage; never NULL). */
const char *kaos_last_error(kaos_handle *h);

/* Device status word: nonzero bits report non-finite state (1) and capacity
 * overflow (2) seen on the device; bit 4 is reserved for a bounded-wait
 * timeout, which no kernel of this build can raise (none waits on another). */
int kaos_get_status(kaos_handle *h, uint32_t *status);

void kaos_destroy(kaos_handle *h);

/*
 * Start-of-step statistics without any device allocation.  This entry point
 * has no counterpart in the reference; it serves callers that cannot call
 * cudaMalloc -- a host running under a fixed device-memory pool of its own,
 * or a process sharing a GPU under an external memory cap.  It bins n ions
 * (field-line q, V||, Vperp1, Vperp2: device arrays; Vperp2 may be NULL only
 * on a 2D grid) into the nq cells bounded by the nq+1 device edges d_qedges
 * (lower boundary first) and the velocity grid vg (host arrays, passed to
 * the kernels by value), and writes the per-cell moments as kaos_get_moments
 * reports them for the first step after a load: d_moments is a device array
 * [11][nq] holding the selectors KAOS_M0 .. KAOS_NQ, d_counts (device, may
 * be NULL) the nq per-cell ion counts.  On a 2D grid an ion whose speed lies
 * outside the grid is left out of the velocity marginals, where a handle
 * keeps the ion's previous bin (the stale-index rule), so the two agree
 * only on the first step after a load.  `stream` is a cudaStream_t (NULL:
 * the default stream).
 *
 * Scratch histograms live in one file-scope device array of at most 512
 * cells x (1 + 3 x 128) counters (about 0.79 MB), held by every GPU that
 * loads the library until the process exits.  nq > 512 or more than 128
 * velocity cells per axis return KAOS_ERR_CAPACITY.  The first call on a
 * device looks up that array's device address (cudaGetSymbolAddress) and
 * the device's SM count with the device current; make that first call on
 * each device before any stream capture begins.  All calls share the
 * array and each clears it first, so calls that overlap on the GPU race:
 * serialise them.
 */
int kaos_moments_noalloc(const kaos_params_c *p, const kaos_vgrid_c *vg,
                         int32_t nq, const double *d_qedges,
                         const double *d_d3x, double nsnormfac,
                         const double *d_q, const double *d_vpar,
                         const double *d_vperp1, const double *d_vperp2,
                         int64_t n, double *d_moments, int64_t *d_counts,
                         void *stream);

/* Library version string. */
const char *kaos_version(void);

#ifdef __cplusplus
}
#endif
#endif /* KAOS_GPU_H */
