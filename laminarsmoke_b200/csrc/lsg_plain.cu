// Plain FP64 reaction step: warp per cell, the reference's algorithm operation
// for operation.  This translation unit is compiled with FMA contraction off
// (-fmad=false) so products and sums round exactly as the CPU code does.
#include "lsg_kernels.h"
#include "lsg_warp_fp64.cuh"

#include <math_constants.h>

namespace lsg {

// solvers/laminarSMOKE/unsteady/chemistry_DI.H:92-235: gather, clip and
// renormalise, integrate, renormalise, scatter; Q is the reactor's QR after
// the solve (chemistry_DI.H:168).
__global__ void __launch_bounds__(kPlainWarpsPerBlock * 32, 1)
plain_warp_kernel(MechLayout L, const unsigned char* __restrict__ mech_gmem, StepOptions o, StepArgs a,
                  int* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ MechLayout sL;
  if (threadIdx.x == 0) sL = L;
  if (!stage_bulk(smem, mech_gmem, L.bytes, &mbar, err)) return;
  const double* Md = (const double*)smem;
  const int* Mi = (const int*)(smem + (size_t)L.n_double * sizeof(double));
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const long cell = (long)blockIdx.x * kPlainWarpsPerBlock + warp;
  if (cell >= a.ncells) return;
  double* wsbase = (double*)(smem + ((L.bytes + 15u) & ~15u)) + (size_t)warp * warp_ws_doubles(L);
  {
    WarpWS W0 = carve_ws(wsbase, L);
    if (lane == 0) {
      W0.SC[0] = 0.; W0.SC[1] = 0.; W0.SC[2] = a.p; W0.SC[3] = o.energy ? 1. : 0.;
      W0.SC[4] = a.rho ? a.rho[cell] : 0.;
    }
    __syncwarp();
  }

  const int NC = L.nc;
  const int ne = NC + 1;
  double yl = 0.;
  if (lane < NC) yl = a.Y[(size_t)lane * a.ld + cell];
  const double Tc = a.T[cell];
  if (lane == NC) yl = Tc;
  double yf = yl;
  int st = 0;
  long long nsteps = 0;
  if (Tc > o.tmin_chem) {
    double y0 = yl;
    if (lane < NC && y0 < 0.) y0 = 0.;
    const double sum = seq_sum(lane < NC ? y0 : 0., NC);
    if (lane < NC) y0 /= sum;
    GearWarp g;
    g.L = &sL;
    g.Md = Md;
    g.Mi = Mi;
    g.ws = wsbase;
    g.W = carve_ws(wsbase, L);
    g.lane = lane;
    g.ne = ne;
    g.active = lane < ne;
    g.alfa2_4 = o.alfa2_4;
    g.alfa2_5 = o.alfa2_5;
    g.maximum_order = (unsigned)o.maximum_order;
    g.max_number_steps = (unsigned)o.max_steps;
    g.abs_tol = o.atol;
    g.rel_tol = o.rtol;
    g.minv = lane < NC ? 0. : o.y_min_T;
    g.maxv = lane < NC ? 1. : o.y_max_T;
    g.b = g.deltab = g.f = g.va = g.vb = g.y = 0.;
    g.eps = 0.;
    g.set_initial_conditions(a.t0, y0);
    const double dtc = a.dt ? a.dt[cell] : a.dt_scalar;
    st = g.solve_to(a.t0 + dtc);
    yf = g.y;
    nsteps = g.cnt[CNT_STEPS];
    if (lane == 0) {
      if (a.Q) a.Q[cell] = g.W.SC[1];
      if (a.counters)
        for (int k = 0; k < NCNT; ++k) a.counters[(size_t)cell * NCNT + k] = g.cnt[k];
    }
  } else if (lane == 0 && a.counters) {
    for (int k = 0; k < NCNT; ++k) a.counters[(size_t)cell * NCNT + k] = 0;
  }
  // solvers/laminarSMOKE/utilities.H:153-200
  const double s = seq_sum(lane < NC ? yf : 0., NC);
  if (lane < NC) {
    yf /= s;
    a.Y[(size_t)lane * a.ld + cell] = yf;
  }
  if (lane == NC && o.energy) a.T[cell] = yf;
  if (lane == 0) {
    if (a.status) a.status[cell] = st;
    if (a.nsteps) a.nsteps[cell] = (int)nsteps;
  }
}

// ---------------------------------------------------------------------------
// DRG-reduced reaction step (solvers/laminarSMOKE/unsteady/chemistry_DRG.H with
// DRG.hpp), one warp per cell.  Per cell above min_T: the directed-relation-graph
// analysis at the cell's state, then the reduced system (the important species
// and T; the other species keep their mass fractions, the dropped reactions have
// zero rate) integrated by a fresh solver from t0 to t0 + dt, the mass fractions
// normalised after the step.
// ---------------------------------------------------------------------------

// Each cell's epsilon: the first band whose temperature is above the cell's; a
// cell above every band keeps the previous analysed cell's epsilon, and cells at
// or below min_T are not analysed (chemistry_DRG.H).  The carry-over runs in cell
// order, so one thread scans the batch.
__global__ void drg_eps_kernel(long ncells, const double* __restrict__ T, DrgArgs d) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double eps = d.epsilon0;
  for (long i = 0; i < ncells; ++i) {
    const double t = T[i];
    if (t > d.min_T)
      for (int b = 0; b < d.nbands; ++b)
        if (t < d.band_T[b]) {
          eps = d.band_eps[b];
          break;
        }
    d.eps[i] = eps;
  }
}

__global__ void __launch_bounds__(kPlainWarpsPerBlock * 32, 1)
drg_warp_kernel(MechLayout L, const unsigned char* __restrict__ mech_gmem, StepOptions o, StepArgs a, DrgArgs d,
                int* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ MechLayout sL;
  if (threadIdx.x == 0) sL = L;
  if (!stage_bulk(smem, mech_gmem, L.bytes, &mbar, err)) return;
  const double* Md = (const double*)smem;
  const int* Mi = (const int*)(smem + (size_t)L.n_double * sizeof(double));
  const MechView M{Md, Mi};
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const long cell = (long)blockIdx.x * kPlainWarpsPerBlock + warp;
  if (cell >= a.ncells) return;
  double* wsbase = (double*)(smem + ((L.bytes + 15u) & ~15u)) + (size_t)warp * drg_ws_doubles(L);
  WarpWS W = carve_ws(wsbase, L);
  if (lane == 0) {
    W.SC[0] = 0.; W.SC[1] = 0.; W.SC[2] = a.p; W.SC[3] = o.energy ? 1. : 0.; W.SC[4] = 0.;
  }
  __syncwarp();
  const int NC = L.nc, NR = L.nr;
  const double Tc = a.T[cell];
  const double om = lane < NC ? a.Y[(size_t)lane * a.ld + cell] : 0.;
  int st = 0, nsp = 0, nrx = 0;
  if (Tc > d.min_T) {
    // ---- analysis (DRG.hpp:150-273): rates at the cell's state, then the search from the key species ----
    rhs_warp<false>(&sL, Md, Mi, wsbase, lane < NC ? om : Tc, Tc);   // W.NET: net rates of progress
    __syncwarp();
    const double eps = d.eps[cell];
    double den = 0.;   // sum_k |nu_ki r_k|, reactions in ascending order
    for (int k = 0; k < NR; ++k) {
      const double nki = lane < NC ? drg_net_nu(M, sL, k, lane) : 0.;
      if (nki != 0.) den += fabs(nki * W.NET[k]);
    }
    int* Qu = (int*)W.J;   // the queue (at most nkey + NC entries; J and G are free until the solve)
    unsigned imp = 0u;
    int qlen = 0;
    for (int t = 0; t < d.nkey; ++t) {
      if (lane == 0) Qu[qlen] = d.key[t];
      ++qlen;
      imp |= 1u << d.key[t];
    }
    __syncwarp();
    for (int head = 0; head < qlen; ++head) {
      const int q = Qu[head];
      const double denq = __shfl_sync(kFull, den, q);
      double num = 0.;
      for (int k = 0; k < NR; ++k) {
        const double nq = drg_net_nu(M, sL, k, q);
        if (nq == 0.) continue;
        const double nkj = lane < NC ? drg_net_nu(M, sL, k, lane) : 0.;
        if (nkj != 0.) num += fabs(nq * W.NET[k]);
      }
      const bool add = lane < NC && !((imp >> lane) & 1u) && num / (1.e-64 + denq) > eps;
      const unsigned m = __ballot_sync(kFull, add);
      if (add) Qu[qlen + __popc(m & ((1u << lane) - 1u))] = lane;   // appended in ascending species order
      qlen += __popc(m);
      imp |= m;
      __syncwarp();
    }
    // a reaction is dropped when one of its species (non-zero net coefficient) was not reached
    int ndrop = 0;
    for (int k = lane; k < NR; k += 32) {
      bool keep = true;
      const int* pp = M.I(L.prod_ptr);
      const int* psp = M.I(L.prod_sp);
      const int* rpp = M.I(L.reac_ptr);
      const int* rsp = M.I(L.reac_sp);
      for (int q = pp[k]; q < pp[k + 1]; ++q) {
        const int s = psp[q];
        if (!((imp >> s) & 1u) && drg_net_nu(M, sL, k, s) != 0.) keep = false;
      }
      for (int q = rpp[k]; q < rpp[k + 1]; ++q) {
        const int s = rsp[q];
        if (!((imp >> s) & 1u) && drg_net_nu(M, sL, k, s) != 0.) keep = false;
      }
      W.DROP[k] = keep ? 0 : 1;
      ndrop += keep ? 0 : 1;
    }
    for (int off = 16; off > 0; off >>= 1) ndrop += __shfl_xor_sync(kFull, ndrop, off);
    __syncwarp();   // the mask is complete before the reduced system reads it
    // ---- the reduced system: lane l < ni owns the l-th important species, lane ni owns T ----
    const int ni = __popc(imp);
    int sp = NC;
    if (lane < ni) {
      unsigned mm = imp;
      for (int t = 0; t < lane; ++t) mm &= mm - 1u;
      sp = __ffs(mm) - 1;
    }
    const int pos = (lane < NC && ((imp >> lane) & 1u)) ? __popc(imp & ((1u << lane) - 1u)) : -1;
    const double ys = __shfl_sync(kFull, om, sp < NC ? sp : 0);
    const double y0 = lane < ni ? ys : (lane == ni ? Tc : 0.);
    GearWarpT<true> g;
    g.L = &sL;
    g.Md = Md;
    g.Mi = Mi;
    g.ws = wsbase;
    g.W = W;
    g.lane = lane;
    g.ne = ni + 1;
    g.active = lane < ni + 1;
    g.drg_ni = ni;
    g.drg_nc = NC;
    g.drg_sp = sp;
    g.drg_pos = pos;
    g.drg_omega = om;
    // a fresh solver object per cell (chemistry_DRG.H): its own order-selection state and step limit
    g.alfa2_4 = 0.8;
    g.alfa2_5 = 0.8;
    g.maximum_order = 5u;
    g.max_number_steps = 500000u;
    if (cell == 0 || !d.first_cell_options_only) {
      g.abs_tol = o.atol;
      g.rel_tol = o.rtol;
      g.minv = lane < ni ? 0. : 200.;
      g.maxv = lane < ni ? 1. : 6000.;
      g.unconstrained = false;
    } else {   // the solver's own defaults (MultiValueSolver.hpp:41-43), no constraints
      g.abs_tol = 1.e-10;
      g.rel_tol = 100. * kMachEpsFloat;
      g.minv = -CUDART_INF;
      g.maxv = CUDART_INF;
      g.unconstrained = true;
    }
    g.b = g.deltab = g.f = g.va = g.vb = g.y = 0.;
    g.eps = 0.;
    g.set_initial_conditions(a.t0, y0);
    const double dtc = a.dt ? a.dt[cell] : a.dt_scalar;
    st = g.solve_to(a.t0 + dtc);
    // ---- scatter: the kept species' start values, the integrated ones, T; normalised ----
    const double yv = __shfl_sync(kFull, g.y, pos >= 0 ? pos : 0);
    const double Tf = __shfl_sync(kFull, g.y, ni);
    double yf = pos >= 0 ? yv : om;
    const double sum = seq_sum(lane < NC ? yf : 0., NC);
    if (lane < NC) {
      yf /= sum;
      a.Y[(size_t)lane * a.ld + cell] = yf;
    }
    if (lane == 0) {
      if (o.energy) a.T[cell] = Tf;
      if (a.Q) a.Q[cell] = W.SC[1];
      if (a.counters)
        for (int k = 0; k < NCNT; ++k) a.counters[(size_t)cell * NCNT + k] = g.cnt[k];
      if (a.nsteps) a.nsteps[cell] = (int)g.cnt[CNT_STEPS];
    }
    nsp = ni;
    nrx = NR - ndrop;
  } else if (lane == 0) {
    if (a.counters)
      for (int k = 0; k < NCNT; ++k) a.counters[(size_t)cell * NCNT + k] = 0;
    if (a.nsteps) a.nsteps[cell] = 0;
  }
  if (lane == 0) {
    if (a.status) a.status[cell] = st;
    if (d.n_species) d.n_species[cell] = nsp;
    if (d.n_reactions) d.n_reactions[cell] = nrx;
  }
}

// Standalone right-hand side, one warp per state (same arithmetic as inside the step).
__global__ void __launch_bounds__(kPlainWarpsPerBlock * 32)
rhs_warp_kernel(MechLayout L, const unsigned char* __restrict__ mech_gmem, long ncells, const double* __restrict__ y,
                double* __restrict__ dy, long ld, double p, int energy, double* qr, int* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ MechLayout sL;
  if (threadIdx.x == 0) sL = L;
  if (!stage_bulk(smem, mech_gmem, L.bytes, &mbar, err)) return;
  const double* Md = (const double*)smem;
  const int* Mi = (const int*)(smem + (size_t)L.n_double * sizeof(double));
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const long cell = (long)blockIdx.x * kPlainWarpsPerBlock + warp;
  if (cell >= ncells) return;
  double* wsbase = (double*)(smem + ((L.bytes + 15u) & ~15u)) + (size_t)warp * warp_ws_doubles(L);
  WarpWS W = carve_ws(wsbase, L);
  if (lane == 0) { W.SC[0] = 0.; W.SC[1] = 0.; W.SC[2] = p; W.SC[3] = energy ? 1. : 0.; W.SC[4] = 0.; }
  __syncwarp();
  const int NC = L.nc;
  const double yl = lane <= NC ? y[(size_t)lane * ld + cell] : 0.;
  const double T = __shfl_sync(kFull, yl, NC);
  const double d = rhs_warp<false>(&sL, Md, Mi, wsbase, yl, T);
  if (lane <= NC) dy[(size_t)lane * ld + cell] = d;
  if (lane == 0 && qr) qr[cell] = W.SC[1];
}

cudaError_t launch_rhs_warp(const MechLayout& L, const unsigned char* mech_gmem, long ncells, const double* y,
                            double* dy, long ld, double p, int energy, double* qr, int* err, cudaStream_t stream) {
  const size_t smem = plain_smem_bytes(L);
  cudaError_t e = cudaFuncSetAttribute(rhs_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const long blocks = (ncells + kPlainWarpsPerBlock - 1) / kPlainWarpsPerBlock;
  rhs_warp_kernel<<<(unsigned)blocks, kPlainWarpsPerBlock * 32, smem, stream>>>(L, mech_gmem, ncells, y, dy, ld, p,
                                                                                 energy, qr, err);
  return cudaGetLastError();
}

size_t plain_smem_bytes(const MechLayout& L) {
  return ((L.bytes + 15u) & ~15u) + (size_t)kPlainWarpsPerBlock * warp_ws_doubles(L) * sizeof(double);
}

cudaError_t upload_gear_plain(const GearConsts& gc) {
  return cudaMemcpyToSymbol(c_gear, &gc, sizeof(GearConsts));
}

cudaError_t launch_plain(const MechLayout& L, const unsigned char* mech_gmem, const StepOptions& o,
                         const StepArgs& a, int* err, cudaStream_t stream) {
  if (a.ncells <= 0) return cudaSuccess;
  const size_t smem = plain_smem_bytes(L);
  cudaError_t e = cudaFuncSetAttribute(plain_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const long blocks = (a.ncells + kPlainWarpsPerBlock - 1) / kPlainWarpsPerBlock;
  plain_warp_kernel<<<(unsigned)blocks, kPlainWarpsPerBlock * 32, smem, stream>>>(L, mech_gmem, o, a, err);
  return cudaGetLastError();
}

cudaError_t launch_drg_eps(long ncells, const double* T, const DrgArgs& d, cudaStream_t stream) {
  if (ncells <= 0) return cudaSuccess;
  drg_eps_kernel<<<1, 32, 0, stream>>>(ncells, T, d);
  return cudaGetLastError();
}

size_t drg_smem_bytes(const MechLayout& L) {
  return ((L.bytes + 15u) & ~15u) + (size_t)kPlainWarpsPerBlock * drg_ws_doubles(L) * sizeof(double);
}

cudaError_t launch_drg_plain(const MechLayout& L, const unsigned char* mech_gmem, const StepOptions& o,
                             const StepArgs& a, const DrgArgs& d, int* err, cudaStream_t stream) {
  if (a.ncells <= 0) return cudaSuccess;
  const size_t smem = drg_smem_bytes(L);
  cudaError_t e = cudaFuncSetAttribute(drg_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = launch_drg_eps(a.ncells, a.T, d, stream);
  if (e != cudaSuccess) return e;
  const long blocks = (a.ncells + kPlainWarpsPerBlock - 1) / kPlainWarpsPerBlock;
  drg_warp_kernel<<<(unsigned)blocks, kPlainWarpsPerBlock * 32, smem, stream>>>(L, mech_gmem, o, a, d, err);
  return cudaGetLastError();
}

}  // namespace lsg
