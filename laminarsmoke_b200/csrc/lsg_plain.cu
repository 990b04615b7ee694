// Plain FP64 reaction step: warp per cell, the reference's algorithm operation
// for operation.  This translation unit is compiled with FMA contraction off
// (-fmad=false) so products and sums round exactly as the CPU code does.
#include "lsg_kernels.h"
#include "lsg_warp_fp64.cuh"

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
  const double d = rhs_warp(&sL, Md, Mi, wsbase, yl, T);
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

}  // namespace lsg
