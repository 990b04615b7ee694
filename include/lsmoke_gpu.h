/*
 * lsmoke_gpu.h -- C ABI of the B200 reaction step for laminarSMOKE.
 *
 * The laminarSMOKE unsteady solvers advance chemistry by operator splitting:
 * every CFD cell is a constant-pressure batch reactor integrated over the
 * cell's time step by the OpenSMOKE++ Gear/BDF multivalue solver.  In the
 * reference this is a serial per-cell loop compiled into the solver
 * (solvers/laminarSMOKE/unsteady/chemistry_DI.H:76-331).  This library
 * replaces that loop with one batched call.  Plain C types only; no CUDA or
 * torch types cross this boundary.
 *
 * Conventions
 *   - Return value 0 = success, negative = library error (lsg_strerror).
 *   - Per-cell ODE outcomes are written to status_out with the reference's
 *     OdeStatus values (math/native-ode-solvers/OdeSolverUtilities.h:83-97):
 *     2 = integrated, 0 = skipped (T <= tmin_chem), -1 max steps, -2 too
 *     strict tolerances, -4 error-test failures, -5 convergence failures,
 *     -6 step too small, -9 illegal initial constraints.  A failed cell keeps
 *     its last accepted state (the reference would hand back stale data).
 *   - Nothing exits, prints or blocks indefinitely.  One context per host
 *     thread per GPU.  Host-pointer calls are synchronous.
 */
#ifndef LSMOKE_GPU_H
#define LSMOKE_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LSG_ABI_VERSION 1

/* library error codes */
#define LSG_OK 0
#define LSG_ERR_ARG -1         /* invalid argument */
#define LSG_ERR_MECH -2        /* mechanism blob could not be read */
#define LSG_ERR_CUDA -3        /* CUDA runtime error */
#define LSG_ERR_NOMEM -4       /* device allocation failed */
#define LSG_ERR_UNSUPPORTED -5 /* option or mechanism size not supported */
#define LSG_ERR_DEVICE -6      /* a kernel reported an internal error flag */
#define LSG_ERR_IO -7          /* file could not be read */
#define LSG_ERR_SCRATCH -8     /* problem does not fit the fixed scratch of lsg_reaction_step_device_noalloc */

/* precision / algorithm forms */
#define LSG_PRECISION_FP64 0   /* plain: the reference method in FP64 */
#define LSG_PRECISION_MIXED 1  /* FP64 rates/residual/error control, FP32 factorisation + FP64 refinement */

/* work decomposition (lsg_options.tile) */
#define LSG_TILE_AUTO 0        /* FP64 -> warp per cell; MIXED -> lane per cell (up to 31 species) */
#define LSG_TILE_WARP 1        /* one warp per cell, the reference's operation order (FP64 only) */
#define LSG_TILE_LANE 2        /* one thread per cell, rounds of RHS / solver / factor kernels over the live cells */
#define LSG_TILE_PERSISTENT 3  /* one thread per cell, one persistent kernel + device work queue */
#define LSG_TILE_BLOCK 4       /* one thread block per cell (any size up to 511 species) */
#define LSG_TILE_GROUP 5       /* one lane group (16 or 32 lanes) per cell from start to finish, the RHS evaluated
                                  by the group inside the solver kernel, persistent grid (up to 31 species) */
/* Mechanisms of 32 to 511 species always run one thread block per cell (the
 * tile is ignored).  The block form factorises in FP64 with LSG_PRECISION_FP64.
 * With LSG_PRECISION_MIXED it inverts G = I - h r0 J on the tensor cores in
 * FP32 (lsg_build_and_invert_g_device: one 128-row tile in tensor memory up to
 * 127 species, an in-place multi-tile inverse in global memory above) and
 * solves with the inverse, refined on the FP64 residual of G until a
 * correction's weighted norm is below 1e-6; a matrix on which the refinement
 * stalls (FP32 cannot hold its conditioning) is refactorised by the FP64 LU.
 * With LSG_TILE_AUTO and autotune = 1 the first step times both
 * factorisations on a sample of the cells and keeps the faster
 * (lsg_ctx_tuning). */

/* counters per cell (lsg_reaction_step_device counters_out layout) */
#define LSG_NCOUNTERS 8        /* steps, rhs, jacobians, factorisations, solves, error-test fails, convergence fails, jacobian rhs */

typedef struct lsg_mech lsg_mech; /* device-resident mechanism tables */
typedef struct lsg_ctx lsg_ctx;   /* per-thread, per-GPU context (stream + buffers) */

/* Solver options.  Defaults (lsg_options_default) are the values the
 * reference tutorials use (run/tutorials/ToroFlames/F3/.../solverOptions:60-64)
 * and the bounds chemistry_DI.H:82-83 sets. */
typedef struct lsg_options {
  double rtol;          /* OdeHomogeneous relTolerance (1e-7) */
  double atol;          /* OdeHomogeneous absTolerance (1e-12) */
  double tmin_chem;     /* minTemperature4Chemistry: cells with T <= tmin_chem are skipped (0) */
  double y_min_T;       /* lower bound on T during integration (200 K) */
  double y_max_T;       /* upper bound on T during integration (6000 K) */
  int max_steps;        /* maximum BDF steps per cell (500000) */
  int full_pivoting;    /* must be 0: partial pivoting (fullPivoting false) */
  int energy;           /* energy equation on (1) / off (0) */
  int precision;        /* LSG_PRECISION_FP64 or LSG_PRECISION_MIXED */
  /* Order-selection state of the reference's solver object: the Gear method
   * lowers alfa2[4], alfa2[5] and its maximum order on every Newton
   * convergence failure and never restores them between cells
   * (MethodGear.hpp:361-385).  Defaults (0.8, 0.8, 5) are a fresh solver. */
  double alfa2_4;
  double alfa2_5;
  int maximum_order;
  int tile;             /* LSG_TILE_* */
  int kernel_timing;    /* 1: time every kernel kind with CUDA events (lsg_ctx_kernel_times) */
  int autotune;         /* 1 with tile LSG_TILE_AUTO: the first step times the candidate forms on a sample of
                           its own cells and keeps the fastest (lsg_ctx_tuning) */
  int jacobian;         /* LSG_JACOBIAN_FD (0, the reference's) or LSG_JACOBIAN_ANALYTIC */
  int reserved[3];
} lsg_options;

/* Newton-matrix Jacobian (lsg_options.jacobian).  The reference always builds
 * it by forward differences, one RHS evaluation per column
 * (KernelDense.hpp:111-193).  LSG_JACOBIAN_ANALYTIC differentiates the rate
 * expressions for the species columns (lsg_jacobian_device) and keeps the
 * temperature column a forward difference; it is used by the lane-per-cell
 * round scheme (LSG_TILE_LANE) of the constant-pressure reactor, the other
 * forms and the constant-volume reactor keep the differences.  It changes the
 * Newton iterates (not their fixed point), so step sequences can differ from
 * the reference's at O(rtol). */
#define LSG_JACOBIAN_FD 0
#define LSG_JACOBIAN_ANALYTIC 1

void lsg_options_default(lsg_options* opt);

/* ---- mechanism --------------------------------------------------------
 * The blob is produced offline from CHEMKIN files by
 * `python -m laminarsmoke_b200.mech compile KIN.CKI THERMO.CKT -o mech.lsmech`
 * (it replaces openSMOKEppCHEMKINPreProcessor + kinetics.xml, which the
 * reference loads at solvers/laminarSMOKE/readOptions.H:62-78).  Every rate
 * form of the compiler is evaluated on the device, the extended PLOG
 * (PLOGMX/PLOGSP) and extended fall-off (LOWMX/LOWSP) forms included. */
int lsg_mech_load_blob(const void* blob, size_t nbytes, int device, lsg_mech** out);
int lsg_mech_load_file(const char* path, int device, lsg_mech** out);
int lsg_mech_info(const lsg_mech* mech, int* nspecies, int* nreactions);
int lsg_mech_destroy(lsg_mech* mech);

/* ---- context ---------------------------------------------------------- */
int lsg_ctx_create(const lsg_mech* mech, const lsg_options* opt, int device, lsg_ctx** out);
int lsg_ctx_set_options(lsg_ctx* ctx, const lsg_options* opt);
int lsg_ctx_destroy(lsg_ctx* ctx);

/* ---- reaction step, host arrays ----------------------------------------
 * Replaces the OpenSMOKE branch of chemistry_DI.H:92-327 (and the
 * SetReactor / SetInitialConditions / Solve / Solution / QR calls it makes,
 * MultiValueSolver.hpp:367-617, BatchReactorHomogeneousConstantPressure.H:60,141).
 *   Y_species  nspecies host pointers, each an array of ncells mass fractions
 *              (OpenFOAM PtrList<volScalarField> layout); updated in place
 *   T          [ncells] temperatures [K]; updated in place when energy is on
 *   p          thermodynamic pressure [Pa]
 *   t0         absolute start time (the initial step size depends on it)
 *   dt         [ncells] per-cell time steps (local time stepping) or NULL
 *   dt_scalar  time step used when dt is NULL
 *   Q_out      [ncells] heat release rate [W/m3] or NULL
 *   status_out [ncells] OdeStatus or NULL
 *   nsteps_out [ncells] accepted BDF steps or NULL */
int lsg_reaction_step(lsg_ctx* ctx, int ncells, int nspecies, double* const* Y_species, double* T, double p,
                      double t0, const double* dt, double dt_scalar, double* Q_out, int* status_out,
                      int* nsteps_out);

/* ---- reaction step, device arrays (state resident in HBM) ---------------
 * Y_dev is species-major: Y_dev[i * ld + cell], ld >= ncells.  All pointers are
 * device pointers; stream is the cudaStream_t the work is enqueued on, used as
 * given (NULL = the legacy default stream; lsg_ctx_stream returns the
 * context's own stream).  Asynchronous: returns after enqueueing.
 * counters_out (optional) receives LSG_NCOUNTERS int64 per cell. */
int lsg_reaction_step_device(lsg_ctx* ctx, int ncells, int nspecies, double* Y_dev, long ld, double* T_dev,
                             double p, double t0, const double* dt_dev, double dt_scalar, double* Q_dev,
                             int* status_dev, int* nsteps_dev, long long* counters_dev, void* stream);

/* ---- successive reaction steps, captured in a CUDA graph -------------------
 * nsteps reaction steps of the same device-resident cells, as a CFD run makes
 * between its flow steps with the state kept in HBM (solvers/laminarSMOKE/
 * unsteady/chemistry_DI.H called once per time step): step k integrates from
 * t0 + k dt to t0 + (k + 1) dt; arrays and conventions as for
 * lsg_reaction_step_device (constant pressure p, scalar dt).  Q_dev and
 * status_dev (optional) hold the last step's values.  The whole sequence is
 * captured once into a CUDA graph on the context's stream and replayed;
 * the context keeps the graph and replays it while every argument stays the
 * same (a changed argument or lsg_ctx_set_options captures anew).  The form
 * whose rounds wait on the host (LSG_TILE_LANE, or the autotuner's choice of
 * it) runs the steps one by one instead.  graph_used (optional) is set to 1
 * when the graph ran.  Ordered after the work already on `stream` and before
 * the work enqueued on it afterwards; asynchronous.  No counterpart in the
 * reference. */
int lsg_reaction_step_sequence_device(lsg_ctx* ctx, int nsteps, int ncells, int nspecies, double* Y_dev, long ld,
                                      double* T_dev, double p, double t0, double dt, double* Q_dev, int* status_dev,
                                      int* graph_used, void* stream);

/* ---- DRG-reduced reaction step ----------------------------------------------
 * Replaces the per-cell loop of solvers/laminarSMOKE/unsteady/chemistry_DRG.H:
 * 86-200 (with unsteady/DRG.hpp: Analysis, PairWiseErrorMatrix,
 * ParsePairWiseErrorMatrix, and the reduced system of
 * BatchReactorHomogeneousConstantPressure.H:253-320).  Per cell above min_T:
 * the directed-relation-graph analysis at the cell's state with the epsilon of
 * the first band whose temperature is above the cell's (a cell above every band
 * keeps the previous analysed cell's epsilon, as the reference's loop does),
 * the reduced system -- the important species and T; the other species keep
 * their mass fractions, the dropped reactions have zero rate -- integrated by a
 * fresh solver from t0 to t0 + dt, the mass fractions normalised after it.  The
 * reference applies the solver options (tolerances; bounds [0, 1] and
 * [200, 6000] K) only when celli == 0, the other cells integrating with the
 * solver's defaults (1e-10 absolute, 100 FLT_EPSILON relative, no bounds):
 * first_cell_options_only = 1 keeps that, 0 gives every cell the options.
 * Cells at or below min_T are left as they are (status 0).  Constant-pressure
 * reactor, FP64: one warp per cell up to 31 species, one thread block per cell
 * above (up to 511).  Options used from the context: rtol, atol, energy.  n_species /
 * n_reactions (optional, device): important species and reactions kept per
 * cell (the reference's drg_important_species / drg_important_reactions
 * fields), 0 for skipped cells. */
#define LSG_DRG_MAX_BANDS 16
typedef struct lsg_drg_options {
  const int* key;           /* host array: key species indices (the DRG "species" list), 1 to nspecies of them */
  int nkey;
  const double* band_T;     /* host arrays of nbands (1..LSG_DRG_MAX_BANDS): temperatures [K] and epsilons */
  const double* band_eps;
  int nbands;
  double epsilon0;          /* epsilon until an analysed cell falls in a band */
  double min_T;             /* minTemperature: cells at or below are not integrated */
  int first_cell_options_only;
} lsg_drg_options;

int lsg_reaction_step_drg_device(lsg_ctx* ctx, int ncells, int nspecies, double* Y_dev, long ld, double* T_dev,
                                 double p, double t0, const double* dt_dev, double dt_scalar,
                                 const lsg_drg_options* drg, double* Q_dev, int* status_dev, int* n_species_dev,
                                 int* n_reactions_dev, long long* counters_dev, void* stream);

/* The same from host fields, as lsg_reaction_step takes them (Y_species: NC
 * pointers to ncells mass fractions; T, dt, Q, status, n_species, n_reactions
 * host arrays of ncells, the outputs optional); synchronous.  Q keeps the
 * caller's values for the cells at or below min_T. */
int lsg_reaction_step_drg(lsg_ctx* ctx, int ncells, int nspecies, double* const* Y_species, double* T, double p,
                          double t0, const double* dt, double dt_scalar, const lsg_drg_options* drg, double* Q,
                          int* status, int* n_species, int* n_reactions);

/* ---- reaction step, constant-volume reactor ------------------------------
 * The branch of chemistry_DI.H taken with constPressureBatchReactor false
 * (:168-203): BatchReactorHomogeneousConstantVolume::SetReactor(V, P, rho)
 * and its Equations (BatchReactorHomogeneousConstantVolume.H:148-199).  Each
 * cell keeps its density rho [kg/m3] (the CFD field rhoCells): the
 * concentrations are rho / MW x_i, dY_i/dt = MW_i R_i / rho and, with the
 * energy equation, dT/dt = (QR + R T sum_i R_i) / (rho cv).  The pressure of
 * the constant-pressure calls has no counterpart (the reactor's P follows
 * from rho and T); every other argument and the pre- and post-processing are
 * those of lsg_reaction_step / lsg_reaction_step_device.  rho may not be NULL. */
int lsg_reaction_step_cv(lsg_ctx* ctx, int ncells, int nspecies, double* const* Y_species, double* T,
                         const double* rho, double t0, const double* dt, double dt_scalar, double* Q_out,
                         int* status_out, int* nsteps_out);
int lsg_reaction_step_cv_device(lsg_ctx* ctx, int ncells, int nspecies, double* Y_dev, long ld, double* T_dev,
                                const double* rho_dev, double t0, const double* dt_dev, double dt_scalar,
                                double* Q_dev, int* status_dev, int* nsteps_dev, long long* counters_dev,
                                void* stream);

/* The context's own stream (a cudaStream_t), for callers without one. */
void* lsg_ctx_stream(lsg_ctx* ctx);

/* Number of kernels this context has enqueued so far (diagnostics; no
 * counterpart in the reference). */
long long lsg_ctx_launches(const lsg_ctx* ctx);

/* Device time per kernel kind, from CUDA events recorded on the launching
 * stream when lsg_options.kernel_timing is set (diagnostics; no counterpart in
 * the reference).  Kinds: 0 RHS, 1 solver advance, 2 compaction, 3 round
 * initialisation (lane-per-cell form), 4 plain warp kernel, 5 persistent lane
 * kernel, 6 block-per-cell kernel (large mechanisms), 7 fused lane-group
 * kernel.  ms[k] total milliseconds, launches[k] timed launches; reset != 0
 * clears the totals after reading.  Waits for the last timed kernel. */
#define LSG_NKERNEL_KINDS 8
int lsg_ctx_kernel_times(lsg_ctx* ctx, double* ms, long long* launches, int nkinds, int reset);

/* Result of the autotuner (lsg_options.autotune; no counterpart in the
 * reference): the chosen tile and its variant (lanes per cell, 16 or 32, for
 * the round scheme; blocks per SM, 4 or 2, for the fused lane-group kernel; 0
 * otherwise) and the measured cells/s of the candidates, in the order round
 * scheme 16 lanes, round scheme 32 lanes, plain warp kernel, persistent lane
 * kernel, fused lane-group kernel at 4 and at 2 blocks per SM (0 for a
 * candidate not tried).  For mechanisms above 31 species with
 * LSG_PRECISION_MIXED the candidates are the block form with FP64 LU factors
 * (rates[0]) and with the tensor-core inverse (rates[1]), timed on one wave of
 * the FP64 form's blocks (at least 256 cells); tile is then LSG_TILE_BLOCK and
 * the variant 1 for the tensor-core inverse, 0 for the FP64 factors.  Returns
 * LSG_ERR_ARG when no tuning has run yet. */
#define LSG_NTUNE_CANDIDATES 6
int lsg_ctx_tuning(const lsg_ctx* ctx, int* tile, int* width, double* rates);

/* Waits for the device, then reads and clears the error flags kernels raised
 * (0 = none).  Returns LSG_ERR_DEVICE when a flag was set. */
int lsg_ctx_check(lsg_ctx* ctx, int* device_flags);

/* ---- reaction step without device allocation ------------------------------
 * No counterpart in the reference: an addition for callers that cannot
 * allocate device memory while they advance the chemistry -- a CFD code that
 * gives all free device memory to its own pool allocator at start-up, or one
 * that keeps cudaMalloc/cudaFree (which synchronise the whole device) out of
 * its time-step loop.  It needs no context: mech (loaded beforehand) and the
 * caller's device arrays, laid out as for lsg_reaction_step_device, are all it
 * takes.  It runs the persistent lane-per-cell kernel (LSG_TILE_PERSISTENT)
 * with its per-cell work space in a fixed array of LSG_NOALLOC_SCRATCH_BYTES
 * that every GPU loading this part of the library keeps until the process
 * exits; as many cells are in flight as that array holds, and any number of
 * cells is processed.
 *   - opt: NULL for the defaults; precision FP64 or MIXED, tile is ignored.
 *   - Mechanisms with more than 31 species do not fit: LSG_ERR_SCRATCH.
 *   - Synchronous: returns when the step has finished on `stream` (NULL = the
 *     legacy default stream).  Loading a mechanism (lsg_mech_load_blob /
 *     lsg_mech_load_file) on a device loads this call's kernels there, commits
 *     the array and looks up its device address, so a caller that hands the
 *     free device memory to its own pool afterwards still has the call work;
 *     the call itself allocates nothing.
 *   - The caller's current device is the same after the call as before it.
 *   - The library caches per-device state (the array's address, uploaded
 *     constants): cudaDeviceReset is not supported while it is loaded.
 *   - All calls on a device share the array and it keeps the previous call's
 *     contents: calls that overlap on the GPU (several streams or host
 *     threads at once) race and must be serialised by the caller. */
#define LSG_NOALLOC_SCRATCH_BYTES (16u << 20)
int lsg_reaction_step_device_noalloc(const lsg_mech* mech, const lsg_options* opt, int ncells, int nspecies,
                                     double* Y_dev, long ld, double* T_dev, double p, double t0, const double* dt_dev,
                                     double dt_scalar, double* Q_dev, int* status_dev, int* nsteps_dev,
                                     long long* counters_dev, void* stream);

/* ---- the mixed-precision factorisation, on its own -------------------------
 * What the mixed-precision block form (LSG_PRECISION_MIXED, 32 to 511
 * species) does where the reference calls KernelDense::BuildAndFactorizeMatrixG
 * (math/native-ode-solvers/KernelDense.hpp:195-220): for nmat Jacobians J_dev
 * [nmat][n][n] (FP64, each column-major: element (i, j) at [j * n + i]) and
 * scalars hr0_dev [nmat], it writes G^-1 of G = I - hr0 J as FP32, column-major,
 * to inv_dev [nmat][n][n].  The inverse is a blocked Gauss-Jordan elimination
 * with partial pivoting whose rank-32 updates run on the tensor cores as split
 * TF32 products (three TF32 products per FP32 product, FP32 accumulation).
 * 1 <= n <= 512 (above 128 the context keeps an FP32 work matrix per block,
 * allocated on the first such call); device pointers; asynchronous on
 * `stream`.  For tests and measurement: the reaction step calls it internally. */
int lsg_build_and_invert_g_device(lsg_ctx* ctx, int nmat, int n, const double* J_dev, const double* hr0_dev,
                                  float* inv_dev, void* stream);

/* ---- analytic Jacobian ------------------------------------------------------
 * J = df/dy of the constant-pressure reactor (BatchReactorHomogeneousConstant
 * Pressure::Equations, :175-223) for ncells states y_dev (species-major
 * [(nspecies + 1) * ld], row nspecies = T), written row-major to J_dev
 * [ncells][n][n] (n = nspecies + 1, element (i, j) = df_i/dy_j at
 * [cell * n * n + i * n + j]).  The species columns are exact derivatives of
 * the rate expressions (Arrhenius, third body, Lindemann/Troe/SRI fall-off,
 * CABR, FORD orders, PLOG/Chebyshev at the given pressure, reverse rates from
 * equilibrium constants or REV); the temperature column is a forward
 * difference with the increment sqrt(eps) max(T, 1).  What the reference
 * would compute in KernelDense::UserDefinedJacobian, which it leaves
 * unimplemented (KernelDense.hpp:96-109); the step uses it with
 * lsg_options.jacobian = LSG_JACOBIAN_ANALYTIC.  Up to 31 species;
 * LSG_ERR_UNSUPPORTED for mechanisms with extended PLOG or fall-off reactions
 * (their constants depend on the concentrations; the step keeps the
 * differences for them). */
int lsg_jacobian_device(lsg_ctx* ctx, int ncells, const double* y_dev, long ld, double p, double* J_dev, void* stream);

/* ---- right-hand side -----------------------------------------------------
 * f(y) of the constant-pressure reactor for ncells states
 * (BatchReactorHomogeneousConstantPressure::Equations, :175-223).  Evaluated
 * by the block form's kernel for more than 31 species or when the context's
 * tile is LSG_TILE_BLOCK, by the warp kernel otherwise.
 * y_dev/dy_dev are species-major [(nspecies+1) * ld], row nspecies = T. */
int lsg_rhs_device(lsg_ctx* ctx, int ncells, const double* y_dev, double* dy_dev, long ld, double p,
                   double* qr_dev, void* stream);

/* ---- output fields beyond Y, T and Q -------------------------------------
 * Source terms of the compact Strang scheme (strangAlgorithm Compact), which
 * replace the field update of solvers/laminarSMOKE/unsteady/chemistry_DI.H:
 * 236-281: from the fields as the step found them (Y0, T0) and the step's
 * result (Yf, Tf, e.g. a copy advanced by lsg_reaction_step_device),
 *   rho = p MW / (R Tf), MW and cp of the mixture at (Yf, Tf),
 *   RR_i = rho (Yf_i - Y0_i) / dt   [kg/m3/s],
 *   RT   = rho cp (Tf - T0) / dt     [W/m3], only with the energy equation on
 *          (lsg_options.energy; RT may be NULL),
 * and zero where dt <= 1e-14.  dt_dev per cell or NULL + dt_scalar (the
 * reference takes the global step tf - t0 here, which equals the cell's step
 * unless local time stepping is on).  All arrays on the device; Y0, Yf and RR
 * species-major [nspecies * ld]. */
int lsg_compact_sources_device(lsg_ctx* ctx, int ncells, int nspecies, const double* Y0_dev, const double* T0_dev,
                               const double* Yf_dev, const double* Tf_dev, long ld, double p, const double* dt_dev,
                               double dt_scalar, double* RR_dev, double* RT_dev, void* stream);

/* Formation-rate output fields (chemistry_DI.H:293-326, outputFormationRates):
 * R_i MW_i [kg/m3/s] of every species at the states (Y, T), written to
 * out_dev [nspecies * ld_out]; the caller picks the species it outputs.  The
 * reference reads the reactor's R() after the solver's last right-hand-side
 * call, which is made at the state the solver returns, i.e. before the
 * driver's renormalisation of Y (a relative change below massFractionsTol =
 * 1e-10).  Uses context-owned scratch of 2 (nspecies + 1) ncells doubles. */
int lsg_formation_rates_device(lsg_ctx* ctx, int ncells, int nspecies, const double* Y_dev, const double* T_dev,
                               long ld, double p, double* out_dev, long ld_out, void* stream);

/* ---- steady solvers: linearised chemical source terms ---------------------
 * What solvers/laminarSMOKE/steady/jacobianEvaluation.H:60-92 computes per
 * cell with linearModel::reactionSourceTerms and ::reactionJacobian
 * (steady/linearModel.H:92-170): the source S_i = R_i MW_i [kg/m3/s] of each
 * species and S_T = QR [W/m3] at omega = max(Y, 0) and T, and the diagonal
 * of its Jacobian J_k = dS_k/dy_k by one forward difference per component
 * (the reference's increment; a perturbed mass fraction is clipped at zero).
 * Outputs, [nspecies + 1][lds] device arrays: S_implicit_k = J_k and
 * S_explicit_k = S_k - J_k y_k, the sourceImplicit / sourceExplicit fields.
 * Pressure per cell (p_dev, the steady solver's p field) or p_scalar when
 * p_dev is NULL.  Uses context-owned scratch of 3 (nspecies + 1) ncells
 * doubles.  LSG_ERR_UNSUPPORTED when the mechanism's tables and the per-thread
 * work arrays do not fit one block's shared memory (about 65 species). */
int lsg_steady_sources_device(lsg_ctx* ctx, int ncells, int nspecies, const double* Y_dev, const double* T_dev,
                              long ld, const double* p_dev, double p_scalar, double* S_implicit_dev,
                              double* S_explicit_dev, long lds, void* stream);

/* The steady solvers' default linearisation, sparseJacobian true
 * (steady/readOptionsSteadyState.H:46): linearModel::reactionJacobianSparse
 * (steady/linearModel.H:172-232).  The same sources S and outputs as
 * lsg_steady_sources_device; the diagonal J_k differs:
 *   species (with species_equations != 0, else 0): the reference's analytic
 *     derivative of the formation rate in omega_k (maps/JacobianSparsityPattern
 *     Map.hpp:427-560) at omega* = max(max(Y, 0), 1e-13), times MW_k -- order
 *     times rate over omega* for the forward and reverse products, the
 *     third-body efficiencies, a 1e-4 difference of the fall-off correction,
 *     and the CABR term;
 *   temperature (with energy_equation != 0, else 0): the forward difference of
 *     the dense path.
 * Same scratch, limits and pressure arguments as lsg_steady_sources_device. */
int lsg_steady_sources_sparse_device(lsg_ctx* ctx, int ncells, int nspecies, const double* Y_dev, const double* T_dev,
                                     long ld, const double* p_dev, double p_scalar, int species_equations,
                                     int energy_equation, double* S_implicit_dev, double* S_explicit_dev, long lds,
                                     void* stream);

/* ---- property update after the step ----------------------------------------
 * What solvers/laminarSMOKE/properties.H:40-190 evaluates per cell after each
 * reaction step, from the mechanism's fitted transport data (a blob compiled
 * with a CHEMKIN transport file; TransportPropertiesMap_CHEMKIN.hpp):
 * mole fractions, cTot, psi, h, mu (Wilke), lambda (Mathur-Saxena), cp, cv,
 * species cp, diffusion coefficients and thermal-diffusion (Soret) terms.
 * Every field pointer may be NULL (not written).  Species fields are
 * species-major [nspecies * ld_out]; Dsoret is [n_thermal_diffusion * ld_out]
 * in the order lsg_mech_transport_info returns. */
typedef struct lsg_property_fields {
  double* X;           /* mole fractions */
  double* cTot;        /* [kmol/m3] */
  double* psi;         /* compressibility MWmix / (R T) [s2/m2] */
  double* mu;          /* dynamic viscosity [kg/m/s] */
  double* lambda;      /* thermal conductivity [W/m/K] (energy or Lewis) */
  double* cp;          /* [J/kg/K] (energy or Lewis) */
  double* cv;          /* [J/kg/K] (energy or Lewis) */
  double* h;           /* [J/kg] */
  double* MWmix;       /* [kg/kmol] */
  double* cp_species;  /* species cp [J/kg/K] (energy or Lewis; the reference's iMassDiffusionInEnergyEquation) */
  double* Dmix;        /* diffusion coefficients [m2/s]; NULL: not evaluated */
  double* Dsoret;      /* Dmix_i theta_i MW_i / MWmix of the light species [m2/s]; needs Dmix */
} lsg_property_fields;

typedef struct lsg_property_options {
  int energy;                  /* energyEquation: lambda, cp, cv and species cp are evaluated */
  int simplified_transport;    /* simplifiedTransportProperties: mu0 (T/300)^0.6759, lambda = mu cp / 0.7 */
  const double* lewis;         /* nspecies Lewis numbers (device for _device, host for the host call), or
                                  NULL: mixture-averaged diffusivities (the reference's MULTICOMPONENT) */
} lsg_property_options;

/* Transport data of a mechanism: has_transport 0/1; n_thermal_diffusion light
 * species (MW <= 20) get Soret terms; their species indices go to indices
 * (NULL, or room for nspecies ints). */
int lsg_mech_transport_info(const lsg_mech* mech, int* has_transport, int* n_thermal_diffusion, int* indices);

/* Device arrays: Y_dev [nspecies * ld], T_dev [ncells], p_dev [ncells] or NULL
 * with p_scalar.  LSG_ERR_UNSUPPORTED when the mechanism has no transport data
 * or more species than one block's shared memory holds (about 260). */
int lsg_properties_device(lsg_ctx* ctx, int ncells, int nspecies, const double* Y_dev, const double* T_dev,
                          long ld, const double* p_dev, double p_scalar, const lsg_property_options* opt,
                          const lsg_property_fields* out_dev, long ld_out, void* stream);

/* The same from host arrays (ld = ld_out = ncells): the inputs go to the device,
 * the kernel runs, the requested fields come back; synchronous.  Uses
 * context-owned device scratch. */
int lsg_properties(lsg_ctx* ctx, int ncells, int nspecies, const double* Y, const double* T, const double* p,
                   double p_scalar, const lsg_property_options* opt, const lsg_property_fields* out);

const char* lsg_strerror(int code);
int lsg_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* LSMOKE_GPU_H */
