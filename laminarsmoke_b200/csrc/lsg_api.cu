// C ABI implementation (include/lsmoke_gpu.h): mechanism upload, contexts,
// buffers, dispatch to the kernel translation units.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/lsmoke_gpu.h"
#include "lsg_kernels.h"
#include "lsg_mech_host.h"

using namespace lsg;

struct lsg_mech {
  HostMech host;
  int device = 0;
  unsigned char* d_buf = nullptr;
  unsigned char* d_tr = nullptr;   // transport table, when the blob has one
};

struct lsg_ctx {
  const lsg_mech* mech = nullptr;
  lsg_options opt{};
  int device = 0;
  cudaStream_t stream = nullptr;
  int* d_err = nullptr;
  long cap = 0;
  double* dY = nullptr;
  double* dT = nullptr;
  double* ddt = nullptr;
  double* dQ = nullptr;
  double* drho = nullptr;       // staged densities of the constant-volume host call
  int* dstatus = nullptr;
  int* dnsteps = nullptr;
  // lane-per-cell (batched) resources
  double* slots = nullptr;
  long nslots = 0;
  int* queue = nullptr;
  int sm_count = 0;
  // round-scheme (lane-per-cell) resources
  void* rstate = nullptr;
  long rcap = 0;
  int rstate_lu64 = -1;
  size_t rcache = 0;            // bytes of the RHS column scratch after the round state
  RoundsPlan rplan{};
  int rplan_lu64 = -1;
  int* nact_host = nullptr;   // pinned
  long long launches = 0;     // kernels enqueued by this context
  // block-per-cell (large mechanism) resources
  double* bws = nullptr;
  float* tcinv_ws = nullptr;    // lsg_build_and_invert_g_device above 128: one FP32 work matrix per block
  size_t tcinv_bytes = 0;
  long bws_blocks = 0;
  long tc_blocks = 0;           // blocks of the tensor-core (mixed-precision) block kernel
  int* bqueue = nullptr;
  int* gqueue = nullptr;        // cell queue of the fused lane-group form
  KernelTimer timer;          // per-kernel device time (lsg_options.kernel_timing)
  // autotuner (lsg_options.autotune)
  bool tuned = false;
  int tuned_tile = 0, tuned_w = 0;
  double tune_rate[LSG_NTUNE_CANDIDATES] = {};
  double* tune_buf = nullptr;   // sample cells: pristine copy and work copy
  long tune_cap = 0;
  int rplan_w = -1;             // lane-group width the round plan was prepared for
  // formation-rate output and steady-solver sources: gathered states and their right-hand sides
  double* frs = nullptr;
  long frs_cap = 0;             // doubles
  // captured step sequence (lsg_reaction_step_sequence_device) and the arguments it was captured for
  cudaGraphExec_t seq_exec = nullptr;
  StepArgs seq_args{};
  int seq_nsteps = 0, seq_tile = -1;
  double seq_dt = 0.;
  cudaEvent_t seq_ev[2] = {nullptr, nullptr};
};

namespace {

std::mutex g_mutex;
bool g_gear_uploaded[64] = {};

// Saves the calling thread's current device and makes it current again when the scope ends.
struct DeviceGuard {
  int dev = -1;
  bool ok = false;
  DeviceGuard() { ok = cudaGetDevice(&dev) == cudaSuccess; }
  ~DeviceGuard() {
    if (ok) cudaSetDevice(dev);
  }
};

GearConsts make_gear_consts() {
  // MethodGear::MemoryAllocationMethod (MethodGear.hpp:125-193)
  GearConsts g{};
  auto fact = [](unsigned n) { unsigned r = 1; for (unsigned k = 2; k <= n; ++k) r *= k; return r; };
  for (int j = 0; j <= 5; ++j) g.Ep[j] = (double)fact(j);
  for (int i = 0; i <= 5; ++i)
    for (int j = 0; j < 5; ++j) g.r[i][j] = 0.;
  g.r[0][0] = 1.;
  g.r[1][0] = 1.;
  for (int j = 2; j <= 5; ++j) {
    g.r[0][j - 1] = (double)fact(j);
    for (int i = 2; i <= j; ++i) g.r[i - 1][j - 1] = double(j) * g.r[i - 1][j - 2] + g.r[i - 2][j - 2];
    g.r[j][j - 1] = 1.;
  }
  double sum = 1.;
  for (int j = 2; j <= 5; ++j) {
    sum += 1. / double(j);
    for (int i = 1; i <= j + 1; ++i) g.r[i - 1][j - 1] /= (fact(j) * sum);
  }
  return g;
}

int ensure_gear(int device) {
  std::lock_guard<std::mutex> lk(g_mutex);
  if (device < 0 || device >= 64) return LSG_ERR_ARG;
  if (g_gear_uploaded[device]) return LSG_OK;
  const GearConsts g = make_gear_consts();
  if (upload_gear_plain(g) != cudaSuccess) return LSG_ERR_CUDA;
  if (upload_gear_batched(g) != cudaSuccess) return LSG_ERR_CUDA;
  if (upload_gear_rounds(g) != cudaSuccess) return LSG_ERR_CUDA;
  if (upload_gear_block(g) != cudaSuccess) return LSG_ERR_CUDA;
  g_gear_uploaded[device] = true;
  return LSG_OK;
}

StepOptions to_step_options(const lsg_options& o) {
  StepOptions s{};
  s.rtol = o.rtol;
  s.atol = o.atol;
  s.tmin_chem = o.tmin_chem;
  s.y_min_T = o.y_min_T;
  s.y_max_T = o.y_max_T;
  s.max_steps = o.max_steps;
  s.energy = o.energy;
  s.alfa2_4 = o.alfa2_4;
  s.alfa2_5 = o.alfa2_5;
  s.maximum_order = o.maximum_order;
  s.jacobian = o.jacobian;
  return s;
}

int validate_options(const lsg_options* o) {
  if (!o) return LSG_ERR_ARG;
  if (!(o->rtol >= 1.e-32) || !(o->atol >= 1.e-32)) return LSG_ERR_ARG;  // MultiValueSolver.hpp:183-199
  if (o->max_steps <= 0) return LSG_ERR_ARG;
  if (!(o->y_min_T < o->y_max_T)) return LSG_ERR_ARG;
  if (o->full_pivoting != 0) return LSG_ERR_UNSUPPORTED;
  if (o->precision != LSG_PRECISION_FP64 && o->precision != LSG_PRECISION_MIXED) return LSG_ERR_ARG;
  if (o->maximum_order < 1 || o->maximum_order > 5) return LSG_ERR_ARG;
  if (o->tile < LSG_TILE_AUTO || o->tile > LSG_TILE_GROUP) return LSG_ERR_ARG;
  if (o->tile == LSG_TILE_WARP && o->precision != LSG_PRECISION_FP64) return LSG_ERR_UNSUPPORTED;
  if (o->jacobian != LSG_JACOBIAN_FD && o->jacobian != LSG_JACOBIAN_ANALYTIC) return LSG_ERR_ARG;
  return LSG_OK;
}

void free_buffers(lsg_ctx* c) {
  cudaFree(c->dY); cudaFree(c->dT); cudaFree(c->ddt); cudaFree(c->dQ); cudaFree(c->dstatus); cudaFree(c->dnsteps);
  cudaFree(c->drho);
  c->dY = c->dT = c->ddt = c->dQ = c->drho = nullptr;
  c->dstatus = c->dnsteps = nullptr;
  c->cap = 0;
}

int ensure_capacity(lsg_ctx* c, long n) {
  if (n <= c->cap) return LSG_OK;
  free_buffers(c);
  const int nc = c->mech->host.layout.nc;
  long cap = n;
  if (cudaMalloc(&c->dY, sizeof(double) * (size_t)nc * cap) != cudaSuccess ||
      cudaMalloc(&c->dT, sizeof(double) * cap) != cudaSuccess ||
      cudaMalloc(&c->ddt, sizeof(double) * cap) != cudaSuccess ||
      cudaMalloc(&c->dQ, sizeof(double) * cap) != cudaSuccess ||
      cudaMalloc(&c->drho, sizeof(double) * cap) != cudaSuccess ||
      cudaMalloc(&c->dstatus, sizeof(int) * cap) != cudaSuccess ||
      cudaMalloc(&c->dnsteps, sizeof(int) * cap) != cudaSuccess) {
    free_buffers(c);
    cudaGetLastError();
    return LSG_ERR_NOMEM;
  }
  c->cap = cap;
  return LSG_OK;
}

int resolve_tile(const lsg_options& o) {
  if (o.tile != LSG_TILE_AUTO) return o.tile;
  return o.precision == LSG_PRECISION_FP64 ? LSG_TILE_WARP : LSG_TILE_LANE;
}

int ensure_batched(lsg_ctx* c, bool lu64) {
  const MechLayout& L = c->mech->host.layout;
  if (!c->sm_count) {
    if (cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess)
      return LSG_ERR_CUDA;
  }
  int bps = 0;
  if (batched_occupancy(L, lu64, &bps) != cudaSuccess || bps <= 0) return LSG_ERR_UNSUPPORTED;
  const long want = (long)c->sm_count * bps * batched_threads_per_block();
  const size_t per = batched_slot_doubles(L, lu64);
  if (c->slots && c->nslots == want) return LSG_OK;
  cudaFree(c->slots);
  c->slots = nullptr;
  c->nslots = 0;
  if (cudaMalloc(&c->slots, sizeof(double) * per * (size_t)want) != cudaSuccess) { cudaGetLastError(); return LSG_ERR_NOMEM; }
  if (!c->queue && cudaMalloc(&c->queue, sizeof(int)) != cudaSuccess) { cudaGetLastError(); return LSG_ERR_NOMEM; }
  c->nslots = want;
  return LSG_OK;
}

// Creates the timing events the first time kernel timing is switched on.
void apply_timing(lsg_ctx* c) {
  if (c->opt.kernel_timing && !c->timer.on) {
    bool ok = true;
    for (cudaEvent_t& e : c->timer.ev)
      if (!e && cudaEventCreate(&e) != cudaSuccess) ok = false;
    c->timer.on = ok;
    if (!ok) cudaGetLastError();
  } else if (!c->opt.kernel_timing) {
    c->timer.on = false;
  }
}

int sm_count(lsg_ctx* c) {
  if (!c->sm_count &&
      cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess)
    return 0;
  return c->sm_count;
}

// One right-hand-side evaluation per cell: the block form's kernel for more
// than 31 species or when the context's tile is LSG_TILE_BLOCK, the warp
// kernel otherwise.
int ensure_block(lsg_ctx* c);
int rhs_dispatch(lsg_ctx* c, long ncells, const double* y, double* dy, long ld, double p, double* qr,
                 cudaStream_t s) {
  const MechLayout& L = c->mech->host.layout;
  if (L.nc + 1 > 32 || c->opt.tile == LSG_TILE_BLOCK) {
    const int r = ensure_block(c);
    if (r != LSG_OK) return r;
    if (launch_rhs_block(L, c->mech->d_buf, ncells, y, dy, ld, p, c->opt.energy, qr, c->bws, c->bws_blocks, s) !=
        cudaSuccess)
      return LSG_ERR_CUDA;
  } else if (launch_rhs_warp(L, c->mech->d_buf, ncells, y, dy, ld, p, c->opt.energy, qr, c->d_err, s) !=
             cudaSuccess) {
    return LSG_ERR_CUDA;
  }
  ++c->launches;
  return LSG_OK;
}

int ensure_rounds(lsg_ctx* c, long n, bool lu64) {
  const MechLayout& L = c->mech->host.layout;
  if (L.nc + 1 > 32) return LSG_ERR_UNSUPPORTED;
  if (!sm_count(c)) return LSG_ERR_CUDA;
  const int w = c->tuned ? c->tuned_w : 0;
  if (c->rplan_lu64 != (int)lu64 || c->rplan_w != w) {
    if (rounds_prepare(L, lu64, c->sm_count, w, &c->rplan) != cudaSuccess) {
      cudaGetLastError();
      return LSG_ERR_UNSUPPORTED;
    }
    c->rplan_lu64 = (int)lu64;
    c->rplan_w = w;
  }
  if (!c->nact_host && cudaMallocHost(&c->nact_host, 2 * sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    return LSG_ERR_NOMEM;
  }
  const size_t cache = rounds_cache_bytes(L, c->rplan);
  if (c->rstate && c->rcap >= n && c->rstate_lu64 == (int)lu64 && c->rcache >= cache) return LSG_OK;
  cudaFree(c->rstate);
  c->rstate = nullptr;
  c->rcap = 0;
  const long cap = (n + 255) & ~255L;
  if (cudaMalloc(&c->rstate, rounds_bytes(L, cap, lu64) + cache) != cudaSuccess) { cudaGetLastError(); return LSG_ERR_NOMEM; }
  c->rcap = cap;
  c->rcache = cache;
  c->rstate_lu64 = (int)lu64;
  return LSG_OK;
}

// Mechanisms with more than 31 species: one block per cell (FP64 factors).
int ensure_block(lsg_ctx* c) {
  const MechLayout& L = c->mech->host.layout;
  if (!sm_count(c)) return LSG_ERR_CUDA;
  if (!c->bws) {
    long nb = 0;
    if (block_plan(L, c->sm_count, false, &nb) != cudaSuccess || nb <= 0) { cudaGetLastError(); return LSG_ERR_UNSUPPORTED; }
    if (cudaMalloc(&c->bws, block_ws_bytes(L) * (size_t)nb) != cudaSuccess) { cudaGetLastError(); return LSG_ERR_NOMEM; }
    if (!c->bqueue && cudaMalloc(&c->bqueue, sizeof(int)) != cudaSuccess) { cudaGetLastError(); return LSG_ERR_NOMEM; }
    c->bws_blocks = nb;
  }
  return LSG_OK;
}

// The block form's buffers and launch plan (FP64 form, and the tensor-core form for mixed precision).
int prepare_large(lsg_ctx* c) {
  const MechLayout& L = c->mech->host.layout;
  const int r = ensure_block(c);
  if (r != LSG_OK) return r;
  if (c->opt.precision == LSG_PRECISION_MIXED && block_tc_eligible(L) && !c->tc_blocks) {
    long t = 0;
    if (block_plan(L, c->sm_count, true, &t) != cudaSuccess || t <= 0) { cudaGetLastError(); return LSG_ERR_UNSUPPORTED; }
    c->tc_blocks = t < c->bws_blocks ? t : c->bws_blocks;
  }
  return LSG_OK;
}

int launch_large(lsg_ctx* c, const StepArgs& a, cudaStream_t s) {
  const MechLayout& L = c->mech->host.layout;
  const int r = prepare_large(c);
  if (r != LSG_OK) return r;
  if (c->timer.used >= KernelTimer::kPairs) {
    cudaStreamSynchronize(s);
    c->timer.collect();
  }
  // mixed precision: the tensor-core inverse (the FP64 form's work space covers its blocks), unless the
  // autotuner measured the FP64 LU factors faster on this context's cells
  const bool tuned_fp64 = c->tuned && c->tuned_tile == LSG_TILE_BLOCK && c->tuned_w == 0;
  const bool tc = c->opt.precision == LSG_PRECISION_MIXED && block_tc_eligible(L) && !tuned_fp64;
  const long nb = tc ? c->tc_blocks : c->bws_blocks;
  c->timer.begin(KT_BLOCK, s);
  if (launch_block(L, c->mech->d_buf, to_step_options(c->opt), a, c->bws, nb, c->bqueue, tc, c->d_err, s) !=
      cudaSuccess)
    return LSG_ERR_CUDA;
  c->timer.end(s);
  c->launches += 1;
  return LSG_OK;
}

int launch_tile(lsg_ctx* c, const StepArgs& a, cudaStream_t s, int tile);

// The autotuner's sample: a pristine copy of the first m cells of the call (Y rows, T, dt) and a work copy
// the trials integrate; t receives the trial arguments over the work copy.
int tune_sample(lsg_ctx* c, const StepArgs& a, cudaStream_t s, long m, StepArgs* t, double** pristine_out,
                double** work_out, size_t* per_out) {
  const int nc = c->mech->host.layout.nc;
  const size_t per = (size_t)nc * m + 2 * (size_t)m;   // Y rows, T, dt
  if (c->tune_cap < m) {
    cudaFree(c->tune_buf);
    c->tune_buf = nullptr;
    c->tune_cap = 0;
    if (cudaMalloc(&c->tune_buf, 2 * per * sizeof(double)) != cudaSuccess) { cudaGetLastError(); return LSG_ERR_NOMEM; }
    c->tune_cap = m;
  }
  double* pristine = c->tune_buf;
  double* work = c->tune_buf + per;
  for (int i = 0; i < nc; ++i)
    if (cudaMemcpyAsync(pristine + (size_t)i * m, a.Y + (size_t)i * a.ld, m * sizeof(double), cudaMemcpyDeviceToDevice,
                        s) != cudaSuccess)
      return LSG_ERR_CUDA;
  if (cudaMemcpyAsync(pristine + (size_t)nc * m, a.T, m * sizeof(double), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return LSG_ERR_CUDA;
  if (a.dt && cudaMemcpyAsync(pristine + (size_t)nc * m + m, a.dt, m * sizeof(double), cudaMemcpyDeviceToDevice,
                              s) != cudaSuccess)
    return LSG_ERR_CUDA;
  *t = a;
  t->ncells = m;
  t->ld = m;
  t->Y = work;
  t->T = work + (size_t)nc * m;
  t->dt = a.dt ? work + (size_t)nc * m + m : nullptr;
  t->Q = nullptr;
  t->status = nullptr;
  t->nsteps = nullptr;
  t->counters = nullptr;
  *pristine_out = pristine;
  *work_out = work;
  *per_out = per;
  return LSG_OK;
}

// Autotuner: times the candidate forms on (a copy of) the first cells of the
// call (up to 262,144) and keeps the fastest for tile LSG_TILE_AUTO.  Candidates: round scheme
// with 16-lane groups (two cells per warp, up to 16 equations) and with 32-lane
// groups, the plain warp kernel (FP64 only) and the persistent lane kernel.
int autotune(lsg_ctx* c, const StepArgs& a, cudaStream_t s) {
  const MechLayout& L = c->mech->host.layout;
  const int nc = L.nc, n = nc + 1;
  (void)nc;
  // The round scheme needs many cells to hide its latency: a small sample would
  // under-rate it, so the sample is up to 262,144 cells (a one-time cost).
  const long m = a.ncells < 262144 ? a.ncells : 262144;
  StepArgs t;
  double *pristine = nullptr, *work = nullptr;
  size_t per = 0;
  const int rs = tune_sample(c, a, s, m, &t, &pristine, &work, &per);
  if (rs != LSG_OK) return rs;
  struct Cand { int tile, w; };
  const Cand cands[LSG_NTUNE_CANDIDATES] = {
      {LSG_TILE_LANE, 16}, {LSG_TILE_LANE, 32}, {LSG_TILE_WARP, 0}, {LSG_TILE_PERSISTENT, 0},
      {LSG_TILE_GROUP, 4}, {LSG_TILE_GROUP, 2}};
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return LSG_ERR_CUDA;
  double best = -1.;
  int besti = -1;
  const bool timing = c->timer.on;
  c->timer.on = false;   // the trial runs are not the caller's kernels
  for (int k = 0; k < LSG_NTUNE_CANDIDATES; ++k) {
    c->tune_rate[k] = 0.;
    const Cand cd = cands[k];
    if (cd.tile == LSG_TILE_LANE && cd.w == 16 && n > 16) continue;
    if (cd.tile == LSG_TILE_WARP && c->opt.precision != LSG_PRECISION_FP64) continue;
    c->tuned = cd.tile == LSG_TILE_LANE || cd.tile == LSG_TILE_GROUP;
    c->tuned_w = cd.w;
    float ms = 0.f;
    for (int rep = 0; rep < 2; ++rep) {   // a 1024-cell run pays the one-time set-up, then the timed run
      if (cudaMemcpyAsync(work, pristine, per * sizeof(double), cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
        c->timer.on = timing;
        return LSG_ERR_CUDA;
      }
      StepArgs tr = t;
      if (rep == 0 && tr.ncells > 1024) tr.ncells = 1024;
      cudaEventRecord(e0, s);
      const int r = launch_tile(c, tr, s, cd.tile);
      cudaEventRecord(e1, s);
      if (r != LSG_OK || cudaEventSynchronize(e1) != cudaSuccess) {
        c->timer.on = timing;
        c->tuned = false;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return r != LSG_OK ? r : LSG_ERR_CUDA;
      }
      cudaEventElapsedTime(&ms, e0, e1);
    }
    c->tune_rate[k] = ms > 0.f ? m / (ms * 1e-3) : 0.;
    if (c->tune_rate[k] > best) { best = c->tune_rate[k]; besti = k; }
  }
  c->timer.on = timing;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (besti < 0) return LSG_ERR_UNSUPPORTED;
  c->tuned = true;
  c->tuned_tile = cands[besti].tile;
  c->tuned_w = cands[besti].w;
  return LSG_OK;
}

// Autotuner for mechanisms above 31 species with mixed precision: the block form with the FP64 LU factors
// (rates[0]) against the block form with the tensor-core inverse (rates[1]), each timed on (a copy of) the
// first min(ncells, slots of the FP64 form) cells, one wave of the FP64 form.  The tensor-core form holds
// more shared memory and TMEM per block, so it runs fewer blocks per SM where the FP64 form fits more;
// which is faster depends on how much of the step the factorisations are.  Keeps tile LSG_TILE_BLOCK with
// width 1 (tensor-core inverse) or 0 (FP64 factors).
int autotune_large(lsg_ctx* c, const StepArgs& a, cudaStream_t s) {
  const MechLayout& L = c->mech->host.layout;
  int r = prepare_large(c);
  if (r != LSG_OK) return r;
  const long m = a.ncells < c->bws_blocks ? a.ncells : c->bws_blocks;
  StepArgs t;
  double *pristine = nullptr, *work = nullptr;
  size_t per = 0;
  r = tune_sample(c, a, s, m, &t, &pristine, &work, &per);
  if (r != LSG_OK) return r;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return LSG_ERR_CUDA;
  const StepOptions so = to_step_options(c->opt);
  for (int k = 0; k < LSG_NTUNE_CANDIDATES; ++k) c->tune_rate[k] = 0.;
  r = LSG_OK;
  for (int k = 0; k < 2 && r == LSG_OK; ++k) {
    const bool tc = k == 1;
    float ms = 0.f;
    if (cudaMemcpyAsync(work, pristine, per * sizeof(double), cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
        cudaEventRecord(e0, s) != cudaSuccess ||
        launch_block(L, c->mech->d_buf, so, t, c->bws, tc ? c->tc_blocks : c->bws_blocks, c->bqueue, tc, c->d_err,
                     s) != cudaSuccess ||
        cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
      cudaGetLastError();
      r = LSG_ERR_CUDA;
      break;
    }
    cudaEventElapsedTime(&ms, e0, e1);
    c->tune_rate[k] = ms > 0.f ? m / (ms * 1e-3) : 0.;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (r != LSG_OK) return r;
  c->tuned = true;
  c->tuned_tile = LSG_TILE_BLOCK;
  c->tuned_w = c->tune_rate[1] > c->tune_rate[0] ? 1 : 0;
  return LSG_OK;
}

// The autotuner, once per context, when tile is LSG_TILE_AUTO and autotune is on.
int maybe_autotune(lsg_ctx* c, const StepArgs& a, cudaStream_t s) {
  const MechLayout& L = c->mech->host.layout;
  if (c->opt.tile != LSG_TILE_AUTO || !c->opt.autotune || c->tuned) return LSG_OK;
  if (L.nc + 1 <= 32) return a.ncells >= 1024 ? autotune(c, a, s) : LSG_OK;
  if (c->opt.precision == LSG_PRECISION_MIXED && block_tc_eligible(L) && a.ncells >= 256)
    return autotune_large(c, a, s);
  return LSG_OK;
}

int launch_step(lsg_ctx* c, const StepArgs& a, cudaStream_t s) {
  const int r = maybe_autotune(c, a, s);
  if (r != LSG_OK) return r;
  const int tile = (c->tuned && c->opt.tile == LSG_TILE_AUTO) ? c->tuned_tile : resolve_tile(c->opt);
  return launch_tile(c, a, s, tile);
}

int launch_tile(lsg_ctx* c, const StepArgs& a, cudaStream_t s, int tile) {
  const MechLayout& L = c->mech->host.layout;
  const StepOptions so = to_step_options(c->opt);
  if (L.nc + 1 > 32 || tile == LSG_TILE_BLOCK) return launch_large(c, a, s);
  if (tile == LSG_TILE_LANE) {
    const bool lu64 = c->opt.precision == LSG_PRECISION_FP64;
    const int r = ensure_rounds(c, a.ncells, lu64);
    if (r != LSG_OK) return r;
    const long max_rounds = 4L * (long)c->opt.max_steps * (L.nc + 9) + 64;
    const cudaError_t e = launch_rounds(c->rplan, L, c->mech->d_buf, so, a, c->rstate, c->rcap, c->nact_host,
                                        max_rounds, c->d_err, s, &c->launches, &c->timer);
    if (e == cudaErrorLaunchTimeout) return LSG_ERR_DEVICE;
    return e == cudaSuccess ? LSG_OK : LSG_ERR_CUDA;
  }
  if (tile == LSG_TILE_GROUP) {
    if (L.nc + 1 > 32) return LSG_ERR_UNSUPPORTED;
    if (!c->gqueue && cudaMalloc(&c->gqueue, sizeof(int)) != cudaSuccess) { cudaGetLastError(); return LSG_ERR_NOMEM; }
    if (!sm_count(c)) return LSG_ERR_CUDA;
    if (c->timer.used >= KernelTimer::kPairs) {
      cudaStreamSynchronize(s);
      c->timer.collect();
    }
    const int mb = (c->tuned && c->tuned_w == 2) ? 2 : 4;   // the autotuner's occupancy variant, else 4 blocks/SM
    c->timer.begin(KT_GROUP, s);
    const cudaError_t e = launch_group(L, c->mech->d_buf, so, a, c->opt.precision == LSG_PRECISION_FP64,
                                       mb == 2 ? 2 : 4, c->gqueue, c->d_err, c->sm_count, s);
    c->timer.end(s);
    if (e == cudaErrorInvalidValue) { cudaGetLastError(); return LSG_ERR_UNSUPPORTED; }
    if (e != cudaSuccess) return LSG_ERR_CUDA;
    c->launches += 1;
    return LSG_OK;
  }
  if (tile == LSG_TILE_WARP) {
    if (L.nc + 1 > 32) return LSG_ERR_UNSUPPORTED;
    if (plain_smem_bytes(L) > 227 * 1024) return LSG_ERR_UNSUPPORTED;
    if (c->timer.used >= KernelTimer::kPairs) {
      cudaStreamSynchronize(s);
      c->timer.collect();
    }
    c->timer.begin(KT_PLAIN, s);
    if (launch_plain(L, c->mech->d_buf, so, a, c->d_err, s) != cudaSuccess) return LSG_ERR_CUDA;
    c->timer.end(s);
    c->launches += 1;
    return LSG_OK;
  }
  const bool lu64 = c->opt.precision == LSG_PRECISION_FP64;
  if (batched_smem_bytes(L, lu64) > 227 * 1024) return LSG_ERR_UNSUPPORTED;
  const int r = ensure_batched(c, lu64);
  if (r != LSG_OK) return r;
  if (cudaMemsetAsync(c->queue, 0, sizeof(int), s) != cudaSuccess) return LSG_ERR_CUDA;
  if (c->timer.used >= KernelTimer::kPairs) {
    cudaStreamSynchronize(s);
    c->timer.collect();
  }
  c->timer.begin(KT_PERSISTENT, s);
  if (launch_batched(L, c->mech->d_buf, so, a, c->slots, c->nslots, nullptr, c->queue, lu64, c->d_err, s) !=
      cudaSuccess)
    return LSG_ERR_CUDA;
  c->timer.end(s);
  c->launches += 1;
  return LSG_OK;
}

}  // namespace

extern "C" {

void lsg_options_default(lsg_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->rtol = 1.e-7;
  o->atol = 1.e-12;
  o->tmin_chem = 0.;
  o->y_min_T = 200.;
  o->y_max_T = 6000.;
  o->max_steps = 500000;
  o->full_pivoting = 0;
  o->energy = 1;
  o->precision = LSG_PRECISION_FP64;
  o->alfa2_4 = 0.8;
  o->alfa2_5 = 0.8;
  o->maximum_order = 5;
}

int lsg_abi_version(void) { return LSG_ABI_VERSION; }

const char* lsg_strerror(int code) {
  switch (code) {
    case LSG_OK: return "success";
    case LSG_ERR_ARG: return "invalid argument";
    case LSG_ERR_MECH: return "mechanism blob could not be read";
    case LSG_ERR_CUDA: return "CUDA runtime error";
    case LSG_ERR_NOMEM: return "device allocation failed";
    case LSG_ERR_UNSUPPORTED: return "option or mechanism size not supported";
    case LSG_ERR_DEVICE: return "a kernel reported an internal error";
    case LSG_ERR_IO: return "file could not be read";
    case LSG_ERR_SCRATCH: return "problem exceeds the fixed no-allocation scratch (at most 31 species)";
    default: return "unknown error";
  }
}

int lsg_mech_load_blob(const void* blob, size_t nbytes, int device, lsg_mech** out) {
  if (!blob || !out) return LSG_ERR_ARG;
  *out = nullptr;
  lsg_mech* m = new (std::nothrow) lsg_mech();
  if (!m) return LSG_ERR_NOMEM;
  std::string err;
  if (!build_mechanism(blob, nbytes, m->host, err)) {
    delete m;
    return err.rfind("unsupported", 0) == 0 ? LSG_ERR_UNSUPPORTED : LSG_ERR_MECH;
  }
  m->device = device;
  if (cudaSetDevice(device) != cudaSuccess) { delete m; cudaGetLastError(); return LSG_ERR_CUDA; }
  // Load the kernel modules now: CUDA loads them lazily, and loading commits device memory (kernel code,
  // the no-allocation entry point's fixed array), which must not wait for the first step call.
  if (ensure_gear(device) != LSG_OK || batched_noalloc_prepare(device) != cudaSuccess) {
    delete m;
    cudaGetLastError();
    return LSG_ERR_CUDA;
  }
  if (cudaMalloc(&m->d_buf, m->host.buffer.size()) != cudaSuccess) { delete m; cudaGetLastError(); return LSG_ERR_NOMEM; }
  if (cudaMemcpy(m->d_buf, m->host.buffer.data(), m->host.buffer.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(m->d_buf);
    delete m;
    return LSG_ERR_CUDA;
  }
  if (m->host.has_transport) {
    const size_t nb = m->host.tbuffer.size();
    if (cudaMalloc(&m->d_tr, nb) != cudaSuccess) {
      cudaGetLastError();
      cudaFree(m->d_buf);
      delete m;
      return LSG_ERR_NOMEM;
    }
    if (cudaMemcpy(m->d_tr, m->host.tbuffer.data(), nb, cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaFree(m->d_tr);
      cudaFree(m->d_buf);
      delete m;
      return LSG_ERR_CUDA;
    }
  }
  *out = m;
  return LSG_OK;
}

int lsg_mech_load_file(const char* path, int device, lsg_mech** out) {
  if (!path || !out) return LSG_ERR_ARG;
  std::ifstream f(path, std::ios::binary);
  if (!f) return LSG_ERR_IO;
  std::vector<char> data((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  return lsg_mech_load_blob(data.data(), data.size(), device, out);
}

int lsg_mech_info(const lsg_mech* m, int* nspecies, int* nreactions) {
  if (!m) return LSG_ERR_ARG;
  if (nspecies) *nspecies = m->host.layout.nc;
  if (nreactions) *nreactions = m->host.layout.nr;
  return LSG_OK;
}

int lsg_mech_destroy(lsg_mech* m) {
  if (!m) return LSG_OK;
  cudaSetDevice(m->device);
  cudaFree(m->d_buf);
  cudaFree(m->d_tr);
  delete m;
  return LSG_OK;
}

int lsg_ctx_create(const lsg_mech* mech, const lsg_options* opt, int device, lsg_ctx** out) {
  if (!mech || !out) return LSG_ERR_ARG;
  *out = nullptr;
  lsg_options o;
  lsg_options_default(&o);
  if (opt) o = *opt;
  const int v = validate_options(&o);
  if (v != LSG_OK) return v;
  if (device != mech->device) return LSG_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) { cudaGetLastError(); return LSG_ERR_CUDA; }
  const int g = ensure_gear(device);
  if (g != LSG_OK) return g;
  lsg_ctx* c = new (std::nothrow) lsg_ctx();
  if (!c) return LSG_ERR_NOMEM;
  c->mech = mech;
  c->opt = o;
  apply_timing(c);
  c->device = device;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&c->d_err, sizeof(int)) != cudaSuccess || cudaMemset(c->d_err, 0, sizeof(int)) != cudaSuccess) {
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    cudaGetLastError();
    return LSG_ERR_CUDA;
  }
  *out = c;
  return LSG_OK;
}

int lsg_ctx_set_options(lsg_ctx* c, const lsg_options* opt) {
  if (!c) return LSG_ERR_ARG;
  const int v = validate_options(opt);
  if (v != LSG_OK) return v;
  c->opt = *opt;
  apply_timing(c);
  c->tuned = false;   // new options: tune again on the next step
  if (c->seq_exec) {  // a captured sequence holds the old options
    cudaStreamSynchronize(c->stream);
    cudaGraphExecDestroy(c->seq_exec);
    c->seq_exec = nullptr;
  }
  return LSG_OK;
}

int lsg_ctx_destroy(lsg_ctx* c) {
  if (!c) return LSG_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  free_buffers(c);
  cudaFree(c->slots);
  cudaFree(c->queue);
  cudaFree(c->rstate);
  cudaFree(c->bws);
  cudaFree(c->tcinv_ws);
  if (c->seq_exec) cudaGraphExecDestroy(c->seq_exec);
  if (c->seq_ev[0]) cudaEventDestroy(c->seq_ev[0]);
  if (c->seq_ev[1]) cudaEventDestroy(c->seq_ev[1]);
  cudaFree(c->bqueue);
  cudaFree(c->gqueue);
  cudaFree(c->tune_buf);
  cudaFree(c->frs);
  if (c->nact_host) cudaFreeHost(c->nact_host);
  cudaFree(c->d_err);
  for (cudaEvent_t& e : c->timer.ev)
    if (e) cudaEventDestroy(e);
  cudaStreamDestroy(c->stream);
  delete c;
  return LSG_OK;
}

void* lsg_ctx_stream(lsg_ctx* c) { return c ? (void*)c->stream : nullptr; }

long long lsg_ctx_launches(const lsg_ctx* c) { return c ? c->launches : -1; }

int lsg_ctx_tuning(const lsg_ctx* c, int* tile, int* width, double* rates) {
  if (!c || !c->tuned || c->opt.tile != LSG_TILE_AUTO || !c->opt.autotune) return LSG_ERR_ARG;
  if (tile) *tile = c->tuned_tile;
  if (width) *width = c->tuned_w;
  if (rates)
    for (int k = 0; k < LSG_NTUNE_CANDIDATES; ++k) rates[k] = c->tune_rate[k];
  return LSG_OK;
}

int lsg_ctx_kernel_times(lsg_ctx* c, double* ms, long long* launches, int nkinds, int reset) {
  if (!c || nkinds < 0) return LSG_ERR_ARG;
  if (cudaSetDevice(c->device) != cudaSuccess) return LSG_ERR_CUDA;
  if (c->timer.used > 0) {
    if (cudaEventSynchronize(c->timer.ev[2 * c->timer.used - 1]) != cudaSuccess) return LSG_ERR_CUDA;
    c->timer.collect();
  }
  for (int k = 0; k < nkinds && k < KT_NKINDS; ++k) {
    if (ms) ms[k] = c->timer.ms[k];
    if (launches) launches[k] = c->timer.n[k];
  }
  if (reset)
    for (int k = 0; k < KT_NKINDS; ++k) {
      c->timer.ms[k] = 0.;
      c->timer.n[k] = 0;
    }
  return LSG_OK;
}

int lsg_ctx_check(lsg_ctx* c, int* flags) {
  if (!c) return LSG_ERR_ARG;
  int h = 0;
  // device-wide: kernels may have been enqueued on caller streams
  if (cudaDeviceSynchronize() != cudaSuccess) return LSG_ERR_CUDA;
  if (cudaMemcpy(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return LSG_ERR_CUDA;
  if (cudaMemset(c->d_err, 0, sizeof(int)) != cudaSuccess) return LSG_ERR_CUDA;
  if (flags) *flags = h;
  return h ? LSG_ERR_DEVICE : LSG_OK;
}

namespace {
// The device-array step of both reactors: rho == nullptr is the constant-pressure reactor at p.
int device_step(lsg_ctx* c, int ncells, int nspecies, double* Y, long ld, double* T, double p, const double* rho,
                double t0, const double* dt, double dt_scalar, double* Q, int* status, int* nsteps,
                long long* counters, void* stream) {
  if (!c || ncells < 0 || !Y || !T || ld < ncells) return LSG_ERR_ARG;
  if (nspecies != c->mech->host.layout.nc) return LSG_ERR_ARG;
  if (!(p > 0.)) return LSG_ERR_ARG;
  if (ncells == 0) return LSG_OK;
  if (cudaSetDevice(c->device) != cudaSuccess) return LSG_ERR_CUDA;
  StepArgs a{};
  a.ncells = ncells;
  a.ld = ld;
  a.Y = Y;
  a.T = T;
  a.dt = dt;
  a.dt_scalar = dt_scalar;
  a.t0 = t0;
  a.p = p;
  a.Q = Q;
  a.status = status;
  a.nsteps = nsteps;
  a.counters = counters;
  a.rho = rho;
  return launch_step(c, a, (cudaStream_t)stream);
}

// The host-array step of both reactors: arrays are staged through the context's device buffers.
int host_step(lsg_ctx* c, int ncells, int nspecies, double* const* Ys, double* T, double p, const double* rho,
              double t0, const double* dt, double dt_scalar, double* Q, int* status, int* nsteps) {
  if (!c || ncells < 0 || !Ys || !T) return LSG_ERR_ARG;
  if (nspecies != c->mech->host.layout.nc) return LSG_ERR_ARG;
  for (int i = 0; i < nspecies; ++i) if (!Ys[i]) return LSG_ERR_ARG;
  if (!(p > 0.)) return LSG_ERR_ARG;
  if (ncells == 0) return LSG_OK;
  if (cudaSetDevice(c->device) != cudaSuccess) return LSG_ERR_CUDA;
  int r = ensure_capacity(c, ncells);
  if (r != LSG_OK) return r;
  cudaStream_t s = c->stream;
  const size_t nb = sizeof(double) * (size_t)ncells;
  for (int i = 0; i < nspecies; ++i)
    if (cudaMemcpyAsync(c->dY + (size_t)i * c->cap, Ys[i], nb, cudaMemcpyHostToDevice, s) != cudaSuccess) return LSG_ERR_CUDA;
  if (cudaMemcpyAsync(c->dT, T, nb, cudaMemcpyHostToDevice, s) != cudaSuccess) return LSG_ERR_CUDA;
  if (dt && cudaMemcpyAsync(c->ddt, dt, nb, cudaMemcpyHostToDevice, s) != cudaSuccess) return LSG_ERR_CUDA;
  if (rho && cudaMemcpyAsync(c->drho, rho, nb, cudaMemcpyHostToDevice, s) != cudaSuccess) return LSG_ERR_CUDA;
  StepArgs a{};
  a.ncells = ncells;
  a.ld = c->cap;
  a.Y = c->dY;
  a.T = c->dT;
  a.dt = dt ? c->ddt : nullptr;
  a.dt_scalar = dt_scalar;
  a.t0 = t0;
  a.p = p;
  a.Q = Q ? c->dQ : nullptr;
  a.status = status ? c->dstatus : nullptr;
  a.nsteps = nsteps ? c->dnsteps : nullptr;
  a.rho = rho ? c->drho : nullptr;
  r = launch_step(c, a, s);
  if (r != LSG_OK) return r;
  for (int i = 0; i < nspecies; ++i)
    if (cudaMemcpyAsync(Ys[i], c->dY + (size_t)i * c->cap, nb, cudaMemcpyDeviceToHost, s) != cudaSuccess) return LSG_ERR_CUDA;
  if (cudaMemcpyAsync(T, c->dT, nb, cudaMemcpyDeviceToHost, s) != cudaSuccess) return LSG_ERR_CUDA;
  if (Q && cudaMemcpyAsync(Q, c->dQ, nb, cudaMemcpyDeviceToHost, s) != cudaSuccess) return LSG_ERR_CUDA;
  if (status && cudaMemcpyAsync(status, c->dstatus, sizeof(int) * ncells, cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return LSG_ERR_CUDA;
  if (nsteps && cudaMemcpyAsync(nsteps, c->dnsteps, sizeof(int) * ncells, cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return LSG_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return LSG_ERR_CUDA;
  int flags = 0;
  return lsg_ctx_check(c, &flags);
}
}  // namespace

int lsg_reaction_step_device(lsg_ctx* c, int ncells, int nspecies, double* Y, long ld, double* T, double p,
                             double t0, const double* dt, double dt_scalar, double* Q, int* status, int* nsteps,
                             long long* counters, void* stream) {
  return device_step(c, ncells, nspecies, Y, ld, T, p, nullptr, t0, dt, dt_scalar, Q, status, nsteps, counters,
                     stream);
}

int lsg_reaction_step_cv_device(lsg_ctx* c, int ncells, int nspecies, double* Y, long ld, double* T,
                                const double* rho, double t0, const double* dt, double dt_scalar, double* Q,
                                int* status, int* nsteps, long long* counters, void* stream) {
  if (!rho) return LSG_ERR_ARG;
  return device_step(c, ncells, nspecies, Y, ld, T, 101325., rho, t0, dt, dt_scalar, Q, status, nsteps, counters,
                     stream);
}

// A sequence of device-resident steps, captured once into a CUDA graph and replayed while the arguments
// stay the same.  Forms whose step waits on the host (the round scheme) run the steps one by one.
int lsg_reaction_step_sequence_device(lsg_ctx* c, int nsteps, int ncells, int nspecies, double* Y, long ld,
                                      double* T, double p, double t0, double dt, double* Q, int* status,
                                      int* graph_used, void* stream) {
  if (graph_used) *graph_used = 0;
  if (!c || nsteps < 0 || ncells < 0 || !Y || !T || ld < ncells || !(p > 0.) || !(dt > 0.)) return LSG_ERR_ARG;
  if (nspecies != c->mech->host.layout.nc) return LSG_ERR_ARG;
  if (nsteps == 0 || ncells == 0) return LSG_OK;
  if (cudaSetDevice(c->device) != cudaSuccess) return LSG_ERR_CUDA;
  const cudaStream_t s = (cudaStream_t)stream;
  StepArgs a{};
  a.ncells = ncells; a.ld = ld; a.Y = Y; a.T = T; a.dt = nullptr; a.dt_scalar = dt; a.t0 = t0; a.p = p;
  a.Q = Q; a.status = status;
  const MechLayout& L = c->mech->host.layout;
  // the form: tuned once (on copies of the cells) when autotuning is on
  {
    const int r = maybe_autotune(c, a, s);
    if (r != LSG_OK) return r;
  }
  int tile = (c->tuned && c->opt.tile == LSG_TILE_AUTO) ? c->tuned_tile : resolve_tile(c->opt);
  if (L.nc + 1 > 32) tile = LSG_TILE_BLOCK;
  if (tile == LSG_TILE_LANE) {   // host-synchronised rounds: no graph
    for (int k = 0; k < nsteps; ++k) {
      a.t0 = t0 + k * dt;
      const int r = launch_tile(c, a, s, tile);
      if (r != LSG_OK) return r;
    }
    return LSG_OK;
  }
  const bool same = c->seq_exec && c->seq_nsteps == nsteps && c->seq_tile == tile && c->seq_dt == dt &&
                    c->seq_args.ncells == a.ncells && c->seq_args.ld == a.ld && c->seq_args.Y == a.Y &&
                    c->seq_args.T == a.T && c->seq_args.t0 == a.t0 && c->seq_args.p == a.p &&
                    c->seq_args.Q == a.Q && c->seq_args.status == a.status;
  if (!c->seq_ev[0]) {
    if (cudaEventCreateWithFlags(&c->seq_ev[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->seq_ev[1], cudaEventDisableTiming) != cudaSuccess)
      return LSG_ERR_CUDA;
  }
  if (!same) {
    if (c->seq_exec) { cudaGraphExecDestroy(c->seq_exec); c->seq_exec = nullptr; }
    // buffers and plans first: nothing is allocated while capturing
    int r = LSG_OK;
    if (tile == LSG_TILE_BLOCK || L.nc + 1 > 32) r = prepare_large(c);
    else if (tile == LSG_TILE_PERSISTENT) r = ensure_batched(c, c->opt.precision == LSG_PRECISION_FP64);
    else if (tile == LSG_TILE_GROUP && !c->gqueue && cudaMalloc(&c->gqueue, sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      r = LSG_ERR_NOMEM;
    }
    if (r == LSG_OK && !sm_count(c)) r = LSG_ERR_CUDA;
    if (r != LSG_OK) return r;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return LSG_ERR_CUDA;
    const bool timing = c->timer.on;
    c->timer.on = false;
    const long long l0 = c->launches;
    if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      c->timer.on = timing;
      cudaGetLastError();
      return LSG_ERR_CUDA;
    }
    for (int k = 0; k < nsteps && r == LSG_OK; ++k) {
      StepArgs ak = a;
      ak.t0 = t0 + k * dt;
      r = launch_tile(c, ak, c->stream, tile);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(c->stream, &graph);
    c->timer.on = timing;
    c->launches = l0;
    if (r != LSG_OK || ec != cudaSuccess || !graph) {
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      return r != LSG_OK ? r : LSG_ERR_CUDA;
    }
    const cudaError_t ei = cudaGraphInstantiate(&c->seq_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) { c->seq_exec = nullptr; cudaGetLastError(); return LSG_ERR_CUDA; }
    c->seq_args = a;
    c->seq_nsteps = nsteps;
    c->seq_tile = tile;
    c->seq_dt = dt;
  }
  // order the replay after the caller's stream and the caller's stream after the replay
  if (cudaEventRecord(c->seq_ev[0], s) != cudaSuccess || cudaStreamWaitEvent(c->stream, c->seq_ev[0], 0) != cudaSuccess)
    return LSG_ERR_CUDA;
  if (cudaGraphLaunch(c->seq_exec, c->stream) != cudaSuccess) return LSG_ERR_CUDA;
  if (cudaEventRecord(c->seq_ev[1], c->stream) != cudaSuccess || cudaStreamWaitEvent(s, c->seq_ev[1], 0) != cudaSuccess)
    return LSG_ERR_CUDA;
  c->launches += (long long)nsteps;
  if (graph_used) *graph_used = 1;
  return LSG_OK;
}

// DRG-reduced step (chemistry_DRG.H:86-200): the plain warp form on the reduced system of each cell.
int lsg_reaction_step_drg_device(lsg_ctx* c, int ncells, int nspecies, double* Y, long ld, double* T, double p,
                                 double t0, const double* dt, double dt_scalar, const lsg_drg_options* drg,
                                 double* Q, int* status, int* n_species, int* n_reactions, long long* counters,
                                 void* stream) {
  if (!c || !drg || ncells < 0 || !Y || !T || ld < ncells || !(p > 0.)) return LSG_ERR_ARG;
  const MechLayout& L = c->mech->host.layout;
  if (nspecies != L.nc) return LSG_ERR_ARG;
  if (!drg->key || drg->nkey < 1 || drg->nkey > L.nc) return LSG_ERR_ARG;
  if (!drg->band_T || !drg->band_eps || drg->nbands < 1 || drg->nbands > LSG_DRG_MAX_BANDS) return LSG_ERR_ARG;
  const bool warp_form = L.nc + 1 <= 32;
  if (warp_form && drg_smem_bytes(L) > 227 * 1024) return LSG_ERR_UNSUPPORTED;
  DrgArgs d{};
  for (int t = 0; t < drg->nkey; ++t) {
    if (drg->key[t] < 0 || drg->key[t] >= L.nc) return LSG_ERR_ARG;
    d.key[t] = drg->key[t];
  }
  d.nkey = drg->nkey;
  for (int b = 0; b < drg->nbands; ++b) {
    d.band_T[b] = drg->band_T[b];
    d.band_eps[b] = drg->band_eps[b];
  }
  d.nbands = drg->nbands;
  d.epsilon0 = drg->epsilon0;
  d.min_T = drg->min_T;
  d.first_cell_options_only = drg->first_cell_options_only != 0;
  d.n_species = n_species;
  d.n_reactions = n_reactions;
  if (ncells == 0) return LSG_OK;
  if (cudaSetDevice(c->device) != cudaSuccess) return LSG_ERR_CUDA;
  if (ncells > c->frs_cap) {   // each cell's epsilon
    const cudaStream_t s0 = (cudaStream_t)stream;
    if (cudaStreamSynchronize(s0) != cudaSuccess) return LSG_ERR_CUDA;
    cudaFree(c->frs);
    c->frs = nullptr;
    c->frs_cap = 0;
    if (cudaMalloc(&c->frs, sizeof(double) * (size_t)ncells) != cudaSuccess) { cudaGetLastError(); return LSG_ERR_NOMEM; }
    c->frs_cap = ncells;
  }
  d.eps = c->frs;
  StepArgs a{};
  a.ncells = ncells;
  a.ld = ld;
  a.Y = Y;
  a.T = T;
  a.dt = dt;
  a.dt_scalar = dt_scalar;
  a.t0 = t0;
  a.p = p;
  a.Q = Q;
  a.status = status;
  a.counters = counters;
  if (warp_form) {
    if (launch_drg_plain(L, c->mech->d_buf, to_step_options(c->opt), a, d, c->d_err, (cudaStream_t)stream) !=
        cudaSuccess) {
      cudaGetLastError();
      return LSG_ERR_CUDA;
    }
  } else {   // one block per cell over the block form's work space
    const int r = prepare_large(c);
    if (r != LSG_OK) return r;
    if (launch_drg_eps(ncells, T, d, (cudaStream_t)stream) != cudaSuccess) {
      cudaGetLastError();
      return LSG_ERR_CUDA;
    }
    const cudaError_t e = launch_drg_block(L, c->mech->d_buf, to_step_options(c->opt), a, d, c->bws,
                                           c->bws_blocks, (cudaStream_t)stream);
    if (e == cudaErrorInvalidValue) { cudaGetLastError(); return LSG_ERR_UNSUPPORTED; }
    if (e != cudaSuccess) { cudaGetLastError(); return LSG_ERR_CUDA; }
  }
  c->launches += 2;
  return LSG_OK;
}

// The DRG-reduced step from host fields: staged through the context's device buffers (the caller's Q is copied
// in first, so that skipped cells keep it, as the device entry leaves it).
int lsg_reaction_step_drg(lsg_ctx* c, int ncells, int nspecies, double* const* Ys, double* T, double p, double t0,
                          const double* dt, double dt_scalar, const lsg_drg_options* drg, double* Q, int* status,
                          int* n_species, int* n_reactions) {
  if (!c || ncells < 0 || !Ys || !T || !drg) return LSG_ERR_ARG;
  if (nspecies != c->mech->host.layout.nc) return LSG_ERR_ARG;
  for (int i = 0; i < nspecies; ++i) if (!Ys[i]) return LSG_ERR_ARG;
  if (!(p > 0.)) return LSG_ERR_ARG;
  if (ncells == 0) return LSG_OK;
  if (cudaSetDevice(c->device) != cudaSuccess) return LSG_ERR_CUDA;
  int r = ensure_capacity(c, ncells);
  if (r != LSG_OK) return r;
  cudaStream_t s = c->stream;
  const size_t nb = sizeof(double) * (size_t)ncells;
  for (int i = 0; i < nspecies; ++i)
    if (cudaMemcpyAsync(c->dY + (size_t)i * c->cap, Ys[i], nb, cudaMemcpyHostToDevice, s) != cudaSuccess) return LSG_ERR_CUDA;
  if (cudaMemcpyAsync(c->dT, T, nb, cudaMemcpyHostToDevice, s) != cudaSuccess) return LSG_ERR_CUDA;
  if (dt && cudaMemcpyAsync(c->ddt, dt, nb, cudaMemcpyHostToDevice, s) != cudaSuccess) return LSG_ERR_CUDA;
  if (Q && cudaMemcpyAsync(c->dQ, Q, nb, cudaMemcpyHostToDevice, s) != cudaSuccess) return LSG_ERR_CUDA;
  int* d_nrx = (int*)c->drho;   // the density buffer is free here (constant pressure)
  r = lsg_reaction_step_drg_device(c, ncells, nspecies, c->dY, c->cap, c->dT, p, t0, dt ? c->ddt : nullptr, dt_scalar,
                                   drg, Q ? c->dQ : nullptr, status ? c->dstatus : nullptr,
                                   n_species ? c->dnsteps : nullptr, n_reactions ? d_nrx : nullptr, nullptr, s);
  if (r != LSG_OK) return r;
  for (int i = 0; i < nspecies; ++i)
    if (cudaMemcpyAsync(Ys[i], c->dY + (size_t)i * c->cap, nb, cudaMemcpyDeviceToHost, s) != cudaSuccess) return LSG_ERR_CUDA;
  if (cudaMemcpyAsync(T, c->dT, nb, cudaMemcpyDeviceToHost, s) != cudaSuccess) return LSG_ERR_CUDA;
  if (Q && cudaMemcpyAsync(Q, c->dQ, nb, cudaMemcpyDeviceToHost, s) != cudaSuccess) return LSG_ERR_CUDA;
  const size_t ni = sizeof(int) * (size_t)ncells;
  if (status && cudaMemcpyAsync(status, c->dstatus, ni, cudaMemcpyDeviceToHost, s) != cudaSuccess) return LSG_ERR_CUDA;
  if (n_species && cudaMemcpyAsync(n_species, c->dnsteps, ni, cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return LSG_ERR_CUDA;
  if (n_reactions && cudaMemcpyAsync(n_reactions, d_nrx, ni, cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return LSG_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return LSG_ERR_CUDA;
  int flags = 0;
  return lsg_ctx_check(c, &flags);
}

int lsg_reaction_step(lsg_ctx* c, int ncells, int nspecies, double* const* Ys, double* T, double p, double t0,
                      const double* dt, double dt_scalar, double* Q, int* status, int* nsteps) {
  return host_step(c, ncells, nspecies, Ys, T, p, nullptr, t0, dt, dt_scalar, Q, status, nsteps);
}

int lsg_reaction_step_cv(lsg_ctx* c, int ncells, int nspecies, double* const* Ys, double* T, const double* rho,
                         double t0, const double* dt, double dt_scalar, double* Q, int* status, int* nsteps) {
  if (!rho) return LSG_ERR_ARG;
  return host_step(c, ncells, nspecies, Ys, T, 101325., rho, t0, dt, dt_scalar, Q, status, nsteps);
}

int lsg_reaction_step_device_noalloc(const lsg_mech* m, const lsg_options* opt, int ncells, int nspecies,
                                     double* Y, long ld, double* T, double p, double t0, const double* dt,
                                     double dt_scalar, double* Q, int* status, int* nsteps, long long* counters,
                                     void* stream) {
  if (!m || ncells < 0 || !Y || !T || ld < ncells) return LSG_ERR_ARG;
  lsg_options o;
  lsg_options_default(&o);
  if (opt) o = *opt;
  o.tile = LSG_TILE_PERSISTENT;
  const int v = validate_options(&o);
  if (v != LSG_OK) return v;
  const MechLayout& L = m->host.layout;
  if (nspecies != L.nc || !(p > 0.)) return LSG_ERR_ARG;
  if (L.nc + 1 > 32) return LSG_ERR_SCRATCH;
  if (ncells == 0) return LSG_OK;
  DeviceGuard dg;   // the caller's current device is restored on every return
  if (!dg.ok || cudaSetDevice(m->device) != cudaSuccess) { cudaGetLastError(); return LSG_ERR_CUDA; }
  const int g = ensure_gear(m->device);
  if (g != LSG_OK) return g;
  const bool lu64 = o.precision == LSG_PRECISION_FP64;
  if (batched_smem_bytes(L, lu64) > 227 * 1024) return LSG_ERR_SCRATCH;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->device) != cudaSuccess) return LSG_ERR_CUDA;
  const long nslots = batched_noalloc_slots(L, lu64, sms);
  if (nslots <= 0) return LSG_ERR_SCRATCH;
  StepArgs a{};
  a.ncells = ncells;
  a.ld = ld;
  a.Y = Y;
  a.T = T;
  a.dt = dt;
  a.dt_scalar = dt_scalar;
  a.t0 = t0;
  a.p = p;
  a.Q = Q;
  a.status = status;
  a.nsteps = nsteps;
  a.counters = counters;
  int flags = 0;
  if (launch_batched_noalloc(L, m->d_buf, to_step_options(o), a, lu64, m->device, nslots, &flags,
                             (cudaStream_t)stream) != cudaSuccess) {
    cudaGetLastError();
    return LSG_ERR_CUDA;
  }
  return flags ? LSG_ERR_DEVICE : LSG_OK;
}

int lsg_build_and_invert_g_device(lsg_ctx* c, int nmat, int n, const double* J, const double* hr0, float* inv,
                                  void* stream) {
  if (!c || nmat < 0 || n < 1 || n > 512 || (nmat > 0 && (!J || !hr0 || !inv))) return LSG_ERR_ARG;
  if (nmat == 0) return LSG_OK;
  if (cudaSetDevice(c->device) != cudaSuccess) return LSG_ERR_CUDA;
  if (!sm_count(c)) return LSG_ERR_CUDA;
  const size_t need = tc_inverse_ws_bytes(n, c->sm_count);
  if (need > c->tcinv_bytes) {
    cudaFree(c->tcinv_ws);
    c->tcinv_ws = nullptr;
    c->tcinv_bytes = 0;
    if (cudaMalloc(&c->tcinv_ws, need) != cudaSuccess) { cudaGetLastError(); return LSG_ERR_NOMEM; }
    c->tcinv_bytes = need;
  }
  if (launch_tc_inverse(nmat, n, J, hr0, inv, c->tcinv_ws, c->sm_count, c->d_err, (cudaStream_t)stream) !=
      cudaSuccess) {
    cudaGetLastError();
    return LSG_ERR_CUDA;
  }
  ++c->launches;
  return LSG_OK;
}

int lsg_jacobian_device(lsg_ctx* c, int ncells, const double* y, long ld, double p, double* J, void* stream) {
  if (!c || ncells < 0 || !y || !J || ld < ncells || !(p > 0.)) return LSG_ERR_ARG;
  if (ncells == 0) return LSG_OK;
  const MechLayout& L = c->mech->host.layout;
  if (L.nc + 1 > 32 || L.n_xplog > 0 || L.n_xfo > 0) return LSG_ERR_UNSUPPORTED;
  if (cudaSetDevice(c->device) != cudaSuccess) return LSG_ERR_CUDA;
  if (!sm_count(c)) return LSG_ERR_CUDA;
  if (launch_jacobian(L, c->mech->d_buf, ncells, y, ld, p, c->opt.energy, J, c->sm_count, c->d_err,
                      (cudaStream_t)stream) != cudaSuccess) {
    cudaGetLastError();
    return LSG_ERR_CUDA;
  }
  ++c->launches;
  return LSG_OK;
}

int lsg_rhs_device(lsg_ctx* c, int ncells, const double* y, double* dy, long ld, double p, double* qr, void* stream) {
  if (!c || ncells < 0 || !y || !dy || ld < ncells || !(p > 0.)) return LSG_ERR_ARG;
  if (ncells == 0) return LSG_OK;
  if (cudaSetDevice(c->device) != cudaSuccess) return LSG_ERR_CUDA;
  return rhs_dispatch(c, ncells, y, dy, ld, p, qr, (cudaStream_t)stream);
}

int lsg_compact_sources_device(lsg_ctx* c, int ncells, int nspecies, const double* Y0, const double* T0,
                               const double* Yf, const double* Tf, long ld, double p, const double* dt,
                               double dt_scalar, double* RR, double* RT, void* stream) {
  if (!c || ncells < 0 || !Y0 || !T0 || !Yf || !Tf || !RR || ld < ncells || !(p > 0.)) return LSG_ERR_ARG;
  if (nspecies != c->mech->host.layout.nc) return LSG_ERR_ARG;
  if (ncells == 0) return LSG_OK;
  if (cudaSetDevice(c->device) != cudaSuccess) return LSG_ERR_CUDA;
  if (launch_compact_sources(c->mech->host.layout, c->mech->d_buf, ncells, Y0, T0, Yf, Tf, ld, p, dt, dt_scalar,
                             c->opt.energy, RR, RT, sm_count(c), (cudaStream_t)stream) != cudaSuccess)
    return LSG_ERR_CUDA;
  ++c->launches;
  return LSG_OK;
}

int lsg_steady_sources_device(lsg_ctx* c, int ncells, int nspecies, const double* Y, const double* T, long ld,
                              const double* p, double p_scalar, double* S_implicit, double* S_explicit, long lds,
                              void* stream) {
  if (!c || ncells < 0 || !Y || !T || !S_implicit || !S_explicit || ld < ncells || lds < ncells) return LSG_ERR_ARG;
  if (!p && !(p_scalar > 0.)) return LSG_ERR_ARG;
  const MechLayout& L = c->mech->host.layout;
  if (nspecies != L.nc) return LSG_ERR_ARG;
  if (ncells == 0) return LSG_OK;
  if (cudaSetDevice(c->device) != cudaSuccess) return LSG_ERR_CUDA;
  const cudaStream_t s = (cudaStream_t)stream;
  const long need = 3L * (L.nc + 1) * ncells;
  if (need > c->frs_cap) {
    if (cudaStreamSynchronize(s) != cudaSuccess) return LSG_ERR_CUDA;
    cudaFree(c->frs);
    c->frs = nullptr;
    c->frs_cap = 0;
    if (cudaMalloc(&c->frs, sizeof(double) * need) != cudaSuccess) { cudaGetLastError(); return LSG_ERR_NOMEM; }
    c->frs_cap = need;
  }
  if (!sm_count(c)) return LSG_ERR_CUDA;
  const cudaError_t e = launch_steady_sources(L, c->mech->d_buf, ncells, Y, T, ld, p, p_scalar, c->frs, S_implicit,
                                              S_explicit, lds, c->sm_count, c->d_err, s);
  if (e == cudaErrorInvalidValue) { cudaGetLastError(); return LSG_ERR_UNSUPPORTED; }
  if (e != cudaSuccess) return LSG_ERR_CUDA;
  ++c->launches;
  return LSG_OK;
}

int lsg_steady_sources_sparse_device(lsg_ctx* c, int ncells, int nspecies, const double* Y, const double* T, long ld,
                                     const double* p, double p_scalar, int species_equations, int energy_equation,
                                     double* S_implicit, double* S_explicit, long lds, void* stream) {
  if (!c || ncells < 0 || !Y || !T || !S_implicit || !S_explicit || ld < ncells || lds < ncells) return LSG_ERR_ARG;
  if (!p && !(p_scalar > 0.)) return LSG_ERR_ARG;
  const MechLayout& L = c->mech->host.layout;
  if (nspecies != L.nc) return LSG_ERR_ARG;
  if (ncells == 0) return LSG_OK;
  if (cudaSetDevice(c->device) != cudaSuccess) return LSG_ERR_CUDA;
  const cudaStream_t s = (cudaStream_t)stream;
  const long need = 3L * (L.nc + 1) * ncells;
  if (need > c->frs_cap) {
    if (cudaStreamSynchronize(s) != cudaSuccess) return LSG_ERR_CUDA;
    cudaFree(c->frs);
    c->frs = nullptr;
    c->frs_cap = 0;
    if (cudaMalloc(&c->frs, sizeof(double) * need) != cudaSuccess) { cudaGetLastError(); return LSG_ERR_NOMEM; }
    c->frs_cap = need;
  }
  if (!sm_count(c)) return LSG_ERR_CUDA;
  const cudaError_t e = launch_steady_sources_sparse(L, c->mech->d_buf, ncells, Y, T, ld, p, p_scalar,
                                                     species_equations ? 1 : 0, energy_equation ? 1 : 0, c->frs,
                                                     S_implicit, S_explicit, lds, c->sm_count, c->d_err, s);
  if (e == cudaErrorInvalidValue) { cudaGetLastError(); return LSG_ERR_UNSUPPORTED; }
  if (e != cudaSuccess) return LSG_ERR_CUDA;
  ++c->launches;
  return LSG_OK;
}

int lsg_formation_rates_device(lsg_ctx* c, int ncells, int nspecies, const double* Y, const double* T, long ld,
                               double p, double* out, long ld_out, void* stream) {
  if (!c || ncells < 0 || !Y || !T || !out || ld < ncells || ld_out < ncells || !(p > 0.)) return LSG_ERR_ARG;
  const MechLayout& L = c->mech->host.layout;
  if (nspecies != L.nc) return LSG_ERR_ARG;
  if (ncells == 0) return LSG_OK;
  if (cudaSetDevice(c->device) != cudaSuccess) return LSG_ERR_CUDA;
  const cudaStream_t s = (cudaStream_t)stream;
  const long need = 2L * (L.nc + 1) * ncells;
  if (need > c->frs_cap) {
    if (cudaStreamSynchronize(s) != cudaSuccess) return LSG_ERR_CUDA;
    cudaFree(c->frs);
    c->frs = nullptr;
    c->frs_cap = 0;
    if (cudaMalloc(&c->frs, sizeof(double) * need) != cudaSuccess) { cudaGetLastError(); return LSG_ERR_NOMEM; }
    c->frs_cap = need;
  }
  double* y = c->frs;
  double* dy = c->frs + (long)(L.nc + 1) * ncells;
  if (launch_gather_state(L.nc, ncells, Y, T, ld, y, sm_count(c), s) != cudaSuccess) return LSG_ERR_CUDA;
  ++c->launches;
  const int r = rhs_dispatch(c, ncells, y, dy, ncells, p, nullptr, s);
  if (r != LSG_OK) return r;
  if (launch_formation_rates(L, c->mech->d_buf, ncells, y, dy, p, out, ld_out, sm_count(c), s) != cudaSuccess)
    return LSG_ERR_CUDA;
  ++c->launches;
  return LSG_OK;
}

int lsg_mech_transport_info(const lsg_mech* m, int* has_transport, int* n_thermal_diffusion, int* indices) {
  if (!m) return LSG_ERR_ARG;
  if (has_transport) *has_transport = m->host.has_transport ? 1 : 0;
  if (n_thermal_diffusion) *n_thermal_diffusion = (int)m->host.iteta.size();
  if (indices)
    for (size_t i = 0; i < m->host.iteta.size(); ++i) indices[i] = m->host.iteta[i];
  return LSG_OK;
}

int lsg_properties_device(lsg_ctx* c, int ncells, int nspecies, const double* Y, const double* T, long ld,
                          const double* p, double p_scalar, const lsg_property_options* opt,
                          const lsg_property_fields* out, long ld_out, void* stream) {
  if (!c || !opt || !out || ncells < 0 || !Y || !T || ld < ncells || ld_out < ncells) return LSG_ERR_ARG;
  if (!p && !(p_scalar > 0.)) return LSG_ERR_ARG;
  if (out->Dsoret && !out->Dmix) return LSG_ERR_ARG;
  const lsg_mech* m = c->mech;
  const MechLayout& L = m->host.layout;
  if (nspecies != L.nc) return LSG_ERR_ARG;
  if (!m->host.has_transport || properties_block(L.nc) == 0) return LSG_ERR_UNSUPPORTED;
  if (ncells == 0) return LSG_OK;
  if (cudaSetDevice(c->device) != cudaSuccess) return LSG_ERR_CUDA;
  PropArgs a{};
  a.ncells = ncells;
  a.Y = Y;
  a.T = T;
  a.ld = ld;
  a.p = p;
  a.p_scalar = p_scalar;
  a.energy = opt->energy ? 1 : 0;
  a.simplified = opt->simplified_transport ? 1 : 0;
  a.lewis = opt->lewis;
  a.X = out->X;
  a.cTot = out->cTot;
  a.psi = out->psi;
  a.mu = out->mu;
  a.lambda = out->lambda;
  a.cp = out->cp;
  a.cv = out->cv;
  a.h = out->h;
  a.MWmix = out->MWmix;
  a.cp_species = out->cp_species;
  a.Dmix = out->Dmix;
  a.Dsoret = out->Dsoret;
  a.ld_out = ld_out;
  if (launch_properties(L, m->d_buf, m->host.tlayout, m->d_tr, a, (cudaStream_t)stream) != cudaSuccess)
    return LSG_ERR_CUDA;
  ++c->launches;
  return LSG_OK;
}

int lsg_properties(lsg_ctx* c, int ncells, int nspecies, const double* Y, const double* T, const double* p,
                   double p_scalar, const lsg_property_options* opt, const lsg_property_fields* out) {
  if (!c || !opt || !out || ncells < 0 || !Y || !T) return LSG_ERR_ARG;
  if (!p && !(p_scalar > 0.)) return LSG_ERR_ARG;
  if (out->Dsoret && !out->Dmix) return LSG_ERR_ARG;
  const lsg_mech* m = c->mech;
  const int nc = m->host.layout.nc;
  if (nspecies != nc) return LSG_ERR_ARG;
  if (!m->host.has_transport || properties_block(nc) == 0) return LSG_ERR_UNSUPPORTED;
  if (ncells == 0) return LSG_OK;
  if (cudaSetDevice(c->device) != cudaSuccess) return LSG_ERR_CUDA;
  const long n = ncells;
  const long nt = (long)m->host.iteta.size();
  // device scratch: inputs, then one slot per requested field
  double* const hp[12] = {out->X, out->cTot, out->psi, out->mu, out->lambda, out->cp, out->cv, out->h,
                          out->MWmix, out->cp_species, out->Dmix, out->Dsoret};
  const long rows[12] = {nc, 1, 1, 1, 1, 1, 1, 1, 1, nc, nc, nt};
  long need = (long)nc * n + 2 * n + nc;
  for (int f = 0; f < 12; ++f)
    if (hp[f]) need += rows[f] * n;
  const cudaStream_t s = c->stream;
  if (need > c->frs_cap) {
    if (cudaStreamSynchronize(s) != cudaSuccess) return LSG_ERR_CUDA;
    cudaFree(c->frs);
    c->frs = nullptr;
    c->frs_cap = 0;
    if (cudaMalloc(&c->frs, sizeof(double) * need) != cudaSuccess) { cudaGetLastError(); return LSG_ERR_NOMEM; }
    c->frs_cap = need;
  }
  double* dY = c->frs;
  double* dT = dY + (long)nc * n;
  double* dp = dT + n;
  double* dLe = dp + n;
  double* cur = dLe + nc;
  double* dev[12] = {};
  for (int f = 0; f < 12; ++f)
    if (hp[f]) {
      dev[f] = cur;
      cur += rows[f] * n;
    }
  if (cudaMemcpyAsync(dY, Y, sizeof(double) * nc * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(dT, T, sizeof(double) * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      (p && cudaMemcpyAsync(dp, p, sizeof(double) * n, cudaMemcpyHostToDevice, s) != cudaSuccess) ||
      (opt->lewis && cudaMemcpyAsync(dLe, opt->lewis, sizeof(double) * nc, cudaMemcpyHostToDevice, s) != cudaSuccess))
    return LSG_ERR_CUDA;
  lsg_property_options o = *opt;
  o.lewis = opt->lewis ? dLe : nullptr;
  const lsg_property_fields fd{dev[0], dev[1], dev[2], dev[3], dev[4],  dev[5],
                               dev[6], dev[7], dev[8], dev[9], dev[10], dev[11]};
  const int r = lsg_properties_device(c, ncells, nspecies, dY, dT, n, p ? dp : nullptr, p_scalar, &o, &fd, n, s);
  if (r != LSG_OK) return r;
  for (int f = 0; f < 12; ++f)
    if (hp[f] && cudaMemcpyAsync(hp[f], dev[f], sizeof(double) * rows[f] * n, cudaMemcpyDeviceToHost, s) != cudaSuccess)
      return LSG_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return LSG_ERR_CUDA;
  return LSG_OK;
}

}  // extern "C"
