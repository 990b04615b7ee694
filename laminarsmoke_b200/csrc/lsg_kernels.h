// Kernel launch interface between the host runtime (lsg_api.cu) and the
// kernel translation units.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

#include "lsg_mech.h"

namespace lsg {

struct StepOptions {
  double rtol, atol, tmin_chem, y_min_T, y_max_T;
  int max_steps, energy;
  double alfa2_4, alfa2_5;
  int maximum_order;
  int jacobian;   // LSG_JACOBIAN_FD or LSG_JACOBIAN_ANALYTIC
};

enum { CNT_STEPS, CNT_RHS, CNT_JAC, CNT_FACT, CNT_SOLVE, CNT_ERRFAIL, CNT_CONVFAIL, CNT_JAC_RHS, NCNT };

// Gear method constants (MethodGear::MemoryAllocationMethod, MethodGear.hpp:125-193),
// computed once on the host and uploaded to each kernel unit's constant bank.
struct GearConsts {
  double r[6][5];
  double Ep[6];
};

constexpr int kPlainWarpsPerBlock = 4;

// Arguments of one reaction-step launch (device pointers).
struct StepArgs {
  long ncells;
  long ld;            // leading dimension of the species-major Y: Y[species * ld + cell]
  double* Y;
  double* T;
  const double* dt;   // per-cell dt or nullptr
  double dt_scalar;
  double t0;
  double p;
  double* Q;          // optional
  int* status;        // optional
  int* nsteps;        // optional
  long long* counters;  // optional [ncells][NCNT]
  const double* rho;  // constant-volume reactor: per-cell density [kg/m3]; nullptr: constant pressure
};

// DRG-reduced step (chemistry_DRG.H, DRG.hpp): key species, (temperature, epsilon) bands, the temperature
// below which cells are skipped, and whether the solver options reach the first cell of the call only.
constexpr int kDrgMaxBands = 16;
struct DrgArgs {
  int key[32];
  int nkey;
  double band_T[kDrgMaxBands];
  double band_eps[kDrgMaxBands];
  int nbands;
  double epsilon0;
  double min_T;
  int first_cell_options_only;
  double* eps;        // [ncells] work: each cell's epsilon (the band scan carries it over between cells)
  int* n_species;     // optional [ncells]: important species (0 for skipped cells)
  int* n_reactions;   // optional [ncells]: reactions kept
};
size_t drg_smem_bytes(const MechLayout& L);
cudaError_t launch_drg_eps(long ncells, const double* T, const DrgArgs& d, cudaStream_t stream);
// more than 31 species: one block per cell over the block form's work space (ws, nblocks of it)
cudaError_t launch_drg_block(const MechLayout& L, const unsigned char* mech_gmem, const StepOptions& o,
                             const StepArgs& a, const DrgArgs& d, double* ws, long nblocks, cudaStream_t stream);
cudaError_t launch_drg_plain(const MechLayout& L, const unsigned char* mech_gmem, const StepOptions& o,
                             const StepArgs& a, const DrgArgs& d, int* err, cudaStream_t stream);

size_t plain_smem_bytes(const MechLayout& L);
cudaError_t upload_gear_plain(const GearConsts& gc);
cudaError_t launch_plain(const MechLayout& L, const unsigned char* mech_gmem, const StepOptions& o,
                         const StepArgs& a, int* err, cudaStream_t stream);
size_t batched_slot_doubles(const MechLayout& L, bool lu64);
size_t batched_smem_bytes(const MechLayout& L, bool lu64);
int batched_threads_per_block();
cudaError_t upload_gear_batched(const GearConsts& gc);
cudaError_t batched_occupancy(const MechLayout& L, bool lu64, int* blocks_per_sm);
cudaError_t launch_batched(const MechLayout& L, const unsigned char* mech_gmem, const StepOptions& o,
                           const StepArgs& a, double* slots, long nslots, const int* order, int* queue, bool lu64,
                           int* err, cudaStream_t stream);
// Block-per-cell step for mechanisms of up to 511 species (lsg_block.cu).
cudaError_t upload_gear_block(const GearConsts& gc);
size_t block_ws_bytes(const MechLayout& L);
// tc: the mixed-precision form with the tensor-core inverse (32 to 128 ODE components; lsg_tc.cuh)
bool block_tc_eligible(const MechLayout& L);
cudaError_t block_plan(const MechLayout& L, int sm_count, bool tc, long* nblocks);
cudaError_t launch_block(const MechLayout& L, const unsigned char* mech_gmem, const StepOptions& o,
                         const StepArgs& a, double* ws, long nblocks, int* queue, bool tc, int* err,
                         cudaStream_t stream);
// G^-1 (FP32, column-major) of G = I - hr0[m] J[m] for nmat column-major FP64 Jacobians of order n <= 512,
// by the tensor-core Gauss-Jordan inverses of the mixed-precision block form (one 128-row tile up to 128,
// the in-place multi-tile inverse above); ws: tc_inverse_ws_bytes(n, sm_count) (unused up to 128).
size_t tc_inverse_ws_bytes(int n, int sm_count);
cudaError_t launch_tc_inverse(int nmat, int n, const double* J, const double* hr0, float* out, float* ws,
                              int sm_count, int* err, cudaStream_t stream);
cudaError_t launch_rhs_block(const MechLayout& L, const unsigned char* mech_gmem, long ncells, const double* y,
                             double* dy, long ld, double p, int energy, double* qr, double* ws, long nblocks,
                             cudaStream_t stream);

// Fixed device scratch of the no-allocation entry point (lsg_batched.cu).
constexpr size_t kNoAllocScratchBytes = (size_t)16 << 20;
cudaError_t batched_noalloc_prepare(int device);
long batched_noalloc_slots(const MechLayout& L, bool lu64, int sm_count);
cudaError_t launch_batched_noalloc(const MechLayout& L, const unsigned char* mech_gmem, const StepOptions& o,
                                   const StepArgs& a, bool lu64, int device, long nslots, int* host_flags,
                                   cudaStream_t stream);

// Optional device timing of each kernel kind with CUDA events recorded on the
// launching stream (lsg_options.kernel_timing).  Pairs are collected after the
// stream has been synchronised.
enum { KT_RHS = 0, KT_ADVANCE, KT_COMPACT, KT_INIT, KT_PLAIN, KT_PERSISTENT, KT_BLOCK, KT_GROUP, KT_NKINDS };
struct KernelTimer {
  static constexpr int kPairs = 64;
  bool on = false;
  cudaEvent_t ev[2 * kPairs] = {};
  int kind[kPairs] = {};
  int used = 0;
  double ms[KT_NKINDS] = {};
  long long n[KT_NKINDS] = {};
  void begin(int k, cudaStream_t s) {
    if (!on || used >= kPairs) return;
    kind[used] = k;
    cudaEventRecord(ev[2 * used], s);
  }
  void end(cudaStream_t s) {
    if (!on || used >= kPairs) return;
    cudaEventRecord(ev[2 * used + 1], s);
    ++used;
  }
  void collect() {   // the stream the events were recorded on has been synchronised
    for (int i = 0; i < used; ++i) {
      float t = 0.f;
      if (cudaEventElapsedTime(&t, ev[2 * i], ev[2 * i + 1]) == cudaSuccess) {
        ms[kind[i]] += t;
        n[kind[i]] += 1;
      }
    }
    used = 0;
  }
};

// Round scheme (lsg_rounds.cu): launch geometry chosen once per context.
struct RoundsPlan {
  bool lu64;
  int w;                       // lanes per cell in the advance kernel (16: two cells per warp; 32)
  size_t rhs_smem, adv_smem;
  unsigned g_rhs, g_adv, g_cmp, g_init;
};
size_t rounds_bytes(const MechLayout& L, long ns, bool lu64);
// Column scratch of the RHS kernel's threads (n doubles per thread of the plan's RHS grid), placed right
// after the rounds_bytes of the state.
size_t rounds_cache_bytes(const MechLayout& L, const RoundsPlan& P);
cudaError_t upload_gear_rounds(const GearConsts& gc);
cudaError_t rounds_prepare(const MechLayout& L, bool lu64, int sm_count, int width, RoundsPlan* plan);
cudaError_t launch_rounds(const RoundsPlan& P, const MechLayout& L, const unsigned char* mech_gmem,
                          const StepOptions& o, const StepArgs& a, void* state, long ns, int* nact_host,
                          long max_rounds, int* err, cudaStream_t stream, long long* launches,
                          KernelTimer* timer);
cudaError_t launch_rhs_warp(const MechLayout& L, const unsigned char* mech_gmem, long ncells, const double* y,
                            double* dy, long ld, double p, int energy, double* qr, int* err, cudaStream_t stream);

// Fused lane-group form (lsg_rounds.cu): one lane group per cell from start to finish, RHS in-kernel;
// min_blocks 4 or 2 blocks per SM (128 or 255 registers a thread); queue: one int
cudaError_t launch_group(const MechLayout& L, const unsigned char* mech_gmem, const StepOptions& o, const StepArgs& a,
                         bool lu64, int min_blocks, int* queue, int* err, int sm_count, cudaStream_t stream);

// Jacobians with analytic species columns (lsg_rounds.cu), up to 31 species; J [ncells][n][n] row-major
cudaError_t launch_jacobian(const MechLayout& L, const unsigned char* mech_gmem, long ncells, const double* y, long ld,
                            double p, int energy, double* J, int sm_count, int* err, cudaStream_t stream);

// source terms and diagonal Jacobian of the steady solvers (lsg_rounds.cu); scratch: 3 (nc + 1) ncells doubles
cudaError_t launch_steady_sources(const MechLayout& L, const unsigned char* mech_gmem, long ncells, const double* Y,
                                  const double* T, long ld, const double* p, double p_scalar, double* scratch,
                                  double* Simp, double* Sexp, long lds, int sm_count, int* err, cudaStream_t stream);

// the steady solvers' default sparse linearisation (lsg_rounds.cu); scratch: 3 (nc + 1) ncells doubles
cudaError_t launch_steady_sources_sparse(const MechLayout& L, const unsigned char* mech_gmem, long ncells,
                                         const double* Y, const double* T, long ld, const double* p, double p_scalar,
                                         int species, int energy, double* scratch, double* Simp, double* Sexp,
                                         long lds, int sm_count, int* err, cudaStream_t stream);

// output fields (lsg_outputs.cu)
cudaError_t launch_compact_sources(const MechLayout& L, const unsigned char* mech_gmem, long ncells,
                                   const double* Y0, const double* T0, const double* Yf, const double* Tf, long ld,
                                   double p, const double* dt, double dt_scalar, int energy, double* RR, double* RT,
                                   int sm_count, cudaStream_t stream);
cudaError_t launch_gather_state(int nc, long ncells, const double* Y, const double* T, long ld, double* y,
                                int sm_count, cudaStream_t stream);
cudaError_t launch_formation_rates(const MechLayout& L, const unsigned char* mech_gmem, long ncells,
                                   const double* y, const double* dy, double p, double* out, long ld_out,
                                   int sm_count, cudaStream_t stream);

// ---- property update after the step (lsg_properties.cu)
struct PropArgs {
  long ncells;
  const double* Y;       // [nc][ld]
  const double* T;       // [ncells]
  long ld;
  const double* p;       // [ncells] or null: p_scalar everywhere
  double p_scalar;
  int energy;            // lambda, cp, cv and the species cp are evaluated
  int simplified;        // mu = mu0 (T/T0)^beta0, lambda = mu cp / Pr0
  const double* lewis;   // [nc] Lewis numbers (device) or null: mixture-averaged diffusivities
  double *X, *cTot, *psi, *mu, *lambda, *cp, *cv, *h, *MWmix;   // null: not written
  double *cp_species, *Dmix, *Dsoret;                            // [nc|n_teta][ld_out], null: not evaluated
  long ld_out;
};
// Largest cells-per-block the property kernel can run for nc species (0: too many species).
int properties_block(int nc);
cudaError_t launch_properties(const MechLayout& L, const unsigned char* mech_gmem, const TransportLayout& TL,
                              const unsigned char* tr_gmem, const PropArgs& a, cudaStream_t stream);

}  // namespace lsg
