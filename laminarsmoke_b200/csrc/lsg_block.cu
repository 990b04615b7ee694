// Block-per-cell reaction step for mechanisms too large for a warp (more than
// 31 species): one thread block integrates one cell, thread k owning ODE
// component k; reactions are spread over the threads.  Persistent grid: blocks
// take cells from a device queue.  All arithmetic FP64; sums are block tree
// reductions.  The method is the one of the plain warp step
// (MultiValueSolver.hpp:367-1328, MethodGear.hpp:79-536, KernelDense.hpp:90-245
// under solvers/openSMOKEpp4laminarSMOKE/math/native-ode-solvers) with the RHS of
// BatchReactorHomogeneousConstantPressure.H:175-223 and the kinetics of
// KineticsMap_CHEMKIN.hpp (kinetic constants recomputed only when T changes,
// :271-297); the mechanism tables are read from global memory (read-only path).
//
// Per-block work space in HBM: Jacobian J and factors G, both n x n stored by
// columns (element (i, j) at [j * n + i], so that the threads of a block, one
// per row, read a column in one coalesced sweep), cached kinetic constants; in shared memory: the Nordsieck arrays, concentrations,
// enthalpies, entropies, net rates and the pivots.
#include "lsg_common.cuh"
#include "lsg_kernels.h"
#include "lsg_tc.cuh"

#include <math_constants.h>

namespace lsg {

static __constant__ GearConsts c_gear_k;

namespace {

constexpr int kBlkMaxN = 512;
// refinement of the mixed-precision solve (GearBlock::solve)
constexpr int kBlkRefineMax = 4;
constexpr double kBlkRefineTol = 1.e-6;

__device__ __forceinline__ double contrib_k(double nu, double v) {
  if (nu == 1.) return v;
  if (nu == 2.) return v + v;
  if (nu == 3.) return v + v + v;
  if (nu == 0.5) return 0.5 * v;
  return nu * v;
}

__device__ __forceinline__ double conc_factor_k(double nu, double c1) {
  if (nu == 1.) return c1;
  if (nu == 2.) return c1 * c1;
  if (nu == 3.) return c1 * c1 * c1;
  if (nu == 0.5) return sqrt(c1);
  return pow(c1, nu);
}

// Block-wide sum; every thread receives the total.  red: BT/32 + 1 doubles.
template <int BT>
__device__ __forceinline__ double bsum(double v, double* red) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(kFull, v, off);
  const int w = threadIdx.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[w] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double s = threadIdx.x < BT / 32 ? red[threadIdx.x] : 0.;
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(kFull, s, off);
    if (threadIdx.x == 0) red[BT / 32] = s;
  }
  __syncthreads();
  return red[BT / 32];
}

// Value of thread src in every thread.
__device__ __forceinline__ double bcast(double v, int src, double* slot) {
  __syncthreads();
  if ((int)threadIdx.x == src) *slot = v;
  __syncthreads();
  return *slot;
}

// Per-block shared work space.
struct BlockShared {
  double* Z;     // [8][BT]
  double* V;     // [8][BT]
  double* C;     // [NC] concentrations
  double* H;     // [NC] h/RT
  double* S;     // [NC] s/R
  double* NET;   // [NR] net rates
  double* X;     // [BT] solve vector
  double* red;   // [BT/32 + 1]
  double* slot;  // [4]: broadcast, cached T, QR, pivot value
  int* PIV;      // [BT]
  int* ival;     // [BT/32 + 1] pivot search scratch
  int* PERM;     // [BT] the factorisation's row interchanges composed: row i of P b is b[PERM[i]]
  // DRG-reduced step only (drg_block_kernel): the reduced <-> full layout exchange and the dropped reactions
  double* DX;           // [BT]
  unsigned char* DROP;  // [NR]
};

template <int BT>
__host__ __device__ inline size_t block_shared_bytes(const MechLayout& L) {
  return sizeof(double) * (16 * BT + 3 * (size_t)L.nc + (size_t)L.nr + BT + BT / 32 + 1 + 4) +
         sizeof(int) * (2 * BT + BT / 32 + 1) + 64;
}

// Threads of the block form: one per ODE component, in whole warpgroups.
__host__ __device__ inline int block_bt(int n) { return n <= 128 ? 128 : (n <= 256 ? 256 : 512); }

// Per-block global work space (doubles).  Up to 128 components: J and G (n x n, column-major), the
// kinetic-constant caches.  Above 128 the mixed-precision form's layout is also covered: J with leading
// dimension Np = the block's threads, the FP64 fallback factors G (n x n), the FP32 inverse (Np x Np),
// the Nordsieck arrays Z and V (8 Np each: they leave shared memory to the inverse's operands), caches.
__host__ __device__ inline size_t round32(size_t x) { return (x + 31) & ~(size_t)31; }
__host__ __device__ inline size_t block_ws_doubles(const MechLayout& L) {
  const size_t n = L.nc + 1;
  const size_t caches = 2 * (size_t)L.nr + 2 * (size_t)(L.n_fo > 0 ? L.n_fo : 1) + 8;
  const size_t fp64 = round32(2 * n * n + caches);
  if (n <= 128) return fp64;
  const size_t np = (size_t)block_bt((int)n);
  const size_t tcl = round32(np * np + round32(n * n) + np * np / 2 + 16 * np + caches);
  return fp64 > tcl ? fp64 : tcl;
}

// Shared memory of the mixed-precision form above 128 components: a persistent head (solve vector,
// reductions, LU pivots, the inverse's pivots, TMEM slot, MMA barrier), then, 1024-byte aligned, one
// region used in turn by the RHS (concentrations, enthalpies, entropies, net rates), by the inverse
// (split-TF32 operands) and by the solves (partial sums).
template <int BT>
__host__ __device__ inline size_t tcl_head_bytes() {
  return sizeof(double) * (BT + BT / 32 + 1 + 4) + sizeof(int) * (4 * BT + BT / 32 + 1 + 4) + 16;
}
template <int BT>
__host__ __device__ inline size_t tcl_union_bytes(const MechLayout& L) {
  const size_t rhs = sizeof(double) * (3 * (size_t)L.nc + L.nr);
  const size_t inv = sizeof(float) * ((2 * (BT / 128) + 2) * (size_t)tc::kOperandFloats + 64 + 4 * tc::kPanel);
  const size_t sol = sizeof(double) * 5 * (size_t)BT;
  size_t m = rhs > inv ? rhs : inv;
  return m > sol ? m : sol;
}
template <int BT>
__host__ __device__ inline size_t tcl_smem_bytes(const MechLayout& L) {
  return tcl_head_bytes<BT>() + 1024 + tcl_union_bytes<BT>(L);
}

// ---------------------------------------------------------------------------
// RHS, block cooperative (thread i < NC owns species i, thread NC owns T).
// ---------------------------------------------------------------------------
template <int BT, bool kDrg = false>
__device__ __noinline__ double rhs_block(const MechLayout& L, const MechView M, const BlockShared& W,
                                         double* __restrict__ karr, double* __restrict__ ukeq,
                                         double* __restrict__ kinf, double* __restrict__ logf, double yl, double T,
                                         double P0, int energy, double rho0) {
  const int tid = threadIdx.x;
  const int NC = L.nc, NR = L.nr;
  const double* MW = M.D(L.mw);
  const double mwl = tid < NC ? MW[tid] : 1.;
  const double u = bsum<BT>(tid < NC ? yl / mwl : 0., W.red);
  const double MWmix = 1. / u;
  double xl = 0.;
  if (tid < NC) { xl = MWmix * yl; xl = xl / mwl; }
  const bool cv = rho0 > 0.;   // constant volume (BatchReactorHomogeneousConstantVolume.H:148-199)
  const double cTot = cv ? rho0 / MWmix : P0 / kRgas / T;
  const double cl = cTot * xl;
  const double rho = cv ? rho0 : cTot * MWmix;
  const double* TM = M.D(L.t_mid);
  const double T2 = T * T, T3 = T2 * T, T4 = T3 * T, uT = 1. / T;
  double hl = 0.;
  if (tid < NC) {
    const double* A = T > TM[tid] ? M.D(L.dh_ht) + 6 * tid : M.D(L.dh_lt) + 6 * tid;
    hl = A[0] + T * A[1] + T2 * A[2] + T3 * A[3] + T4 * A[4] + uT * A[5];
    W.C[tid] = cl;
    W.H[tid] = hl;
  }
  const double T_old = W.slot[1];
  const bool recalc = fabs(T - T_old) / T > 0.;
  if (recalc && tid < NC) {
    const double logT = log(T);
    const double* A = T > TM[tid] ? M.D(L.ds_ht) + 6 * tid : M.D(L.ds_lt) + 6 * tid;
    W.S[tid] = A[0] * logT + T * A[1] + T2 * A[2] + T3 * A[3] + T4 * A[4] + A[5];
  }
  __syncthreads();
  if (tid == 0) W.slot[1] = T;
  if (recalc) {
    const double logT = log(T);
    const double lP = log(101325. / kRgas / T);
    const double* lnA = M.D(L.lnA);
    const double* beta = M.D(L.beta);
    const double* eor = M.D(L.eor);
    const double* dnu = M.D(L.dnu);
    const int* sgn = M.I(L.a_sign);
    const int* rk = M.I(L.rev_kind);
    const int* rs = M.I(L.rev_slot);
    const int* rp = M.I(L.reac_ptr);
    const int* rsp = M.I(L.reac_sp);
    const double* rnu = M.D(L.reac_nu);
    const int* pp = M.I(L.prod_ptr);
    const int* psp = M.I(L.prod_sp);
    const double* pnu = M.D(L.prod_nu);
    for (int j = tid; j < NR; j += BT) {
      double k = exp(lnA[j] + beta[j] * logT - eor[j] * uT);
      if (sgn[j] < 0) k *= -1.;
      karr[j] = k;
      const int kind = rk[j];
      if (kind == 1) {
        // StoichiometricMap::ReactionEnthalpyAndEntropy: species order, reactant first
        double dh = 0., ds = 0.;
        int a = rp[j], b = pp[j];
        const int ae = rp[j + 1], be = pp[j + 1];
        while (a < ae || b < be) {
          const int sa = a < ae ? rsp[a] : (1 << 30);
          const int sb = b < be ? psp[b] : (1 << 30);
          if (sa <= sb) {
            dh -= contrib_k(rnu[a], W.H[sa]);
            ds -= contrib_k(rnu[a], W.S[sa]);
            ++a;
          } else {
            dh += contrib_k(pnu[b], W.H[sb]);
            ds += contrib_k(pnu[b], W.S[sb]);
            ++b;
          }
        }
        ukeq[j] = exp(-ds + dh - lP * dnu[j]);
      } else if (kind == 2) {
        const int s = rs[j];
        ukeq[j] = exp(M.D(L.rev_lnA)[s] + M.D(L.rev_beta)[s] * logT - M.D(L.rev_eor)[s] * uT);
      }
    }
    const int* ft = M.I(L.fo_type);
    for (int k = tid; k < L.n_fo; k += BT) {
      kinf[k] = exp(M.D(L.fo_lnA)[k] + M.D(L.fo_beta)[k] * logT - M.D(L.fo_eor)[k] * uT);
      const double a = M.D(L.fo_a)[k], b = M.D(L.fo_b)[k], c = M.D(L.fo_c)[k], d = M.D(L.fo_d)[k];
      if (ft[k] == 1) {
        const double v = (d != 0.) ? (1. - a) * exp(-T / b) + a * exp(-T / c) + exp(-d / T)
                                   : (1. - a) * exp(-T / b) + a * exp(-T / c);
        logf[k] = (v < 1.e-300) ? -300. : log10(v);
      } else if (ft[k] == 2) {
        logf[k] = a * exp(-b / T) + exp(-T / c);
      } else {
        logf[k] = 0.;
      }
    }
  }
  if (L.n_plog > 0 || L.n_cheb > 0) {
    // pressure-logarithmic and Chebyshev reactions: k depends on P too, so every call
    // (KineticsMap_CHEMKIN.hpp:1332-1348)
    const double Pk = cv ? cTot * kRgas * T : P0;
    const double logTk = log(T);
    const int* prx = M.I(L.plog_rxn);
    __syncthreads();   // after the Arrhenius values other threads wrote above
    for (int k = tid; k < L.n_plog; k += BT) karr[prx[k]] = plog_k(M, L, k, T, logTk, Pk);
    const int* crx = M.I(L.cheb_rxn);
    for (int k = tid; k < L.n_cheb; k += BT) karr[crx[k]] = cheb_k(M, L, k, T, Pk);
  }
  const double cTotSum = bsum<BT>(cl, W.red);   // also orders the cache writes above before their reads
  {
    const int* tbs = M.I(L.tb_slot);
    const int* fos = M.I(L.fo_slot);
    const int* rk = M.I(L.rev_kind);
    const int* rp = M.I(L.reac_ptr);
    const int* rsp = M.I(L.reac_sp);
    const double* rnu = M.D(L.reac_nu);
    const int* op = M.I(L.ford_ptr);     // forward rate-law orders (FORD, else the coefficients)
    const int* osp = M.I(L.ford_sp);
    const double* onu = M.D(L.ford_val);
    const int* pp = M.I(L.prod_ptr);
    const int* psp = M.I(L.prod_sp);
    const double* pnu = M.D(L.prod_nu);
    for (int j = tid; j < NR; j += BT) {
      double kArr = karr[j];
      if (L.n_xplog > 0) {   // extended PLOG, every call: k depends on the concentrations (KineticsMap_CHEMKIN.hpp:1662-1670)
        const int xs = M.I(L.xplog_slot)[j];
        if (xs >= 0) kArr = xplog_k(M, L, xs, T, log(T), cv ? cTot * kRgas * T : P0, cTotSum, [&](int k) { return W.C[k]; });
      }
      double kMod = kArr;
      const int tb = tbs[j];
      if (tb >= 0) {
        double Mc = cTotSum;
        const int* tp = M.I(L.tb_ptr);
        const int* ts = M.I(L.tb_sp);
        const double* te = M.D(L.tb_eff);
        for (int q = tp[tb]; q < tp[tb + 1]; ++q) Mc += W.C[ts[q]] * te[q];
        kMod *= Mc;
      }
      const int fo = fos[j];
      if (fo >= 0) {
        double Mc;
        const int single = M.I(L.fo_single)[fo];
        if (single < 0) {
          Mc = cTotSum;
          const int* fp = M.I(L.fo_ptr);
          const int* fs = M.I(L.fo_sp);
          const double* fe = M.D(L.fo_eff);
          for (int q = fp[fo]; q < fp[fo + 1]; ++q) Mc += W.C[fs[q]] * fe[q];
        } else {
          Mc = W.C[single] + 1.e-16;
        }
        const double kInf = kinf[fo];
        const double lF = logf[fo];
        const double Pr = kArr * Mc / kInf;
        const bool cabr = M.I(L.fo_cabr)[fo] != 0;
        double wF = 1.;
        const int ty = M.I(L.fo_type)[fo];
        if (ty == 1) {
          double qq;
          if (Pr > 1.e-32 || cabr) {
            const double nTroe = 0.75 - 1.27 * lF;
            const double cTroe = -0.4 - 0.67 * lF;
            const double sTroe = log10(Pr) + cTroe;
            qq = sTroe / (nTroe - 0.14 * sTroe);
          } else {
            qq = 1. / 0.14;
          }
          wF = pow(10., lF / (1. + qq * qq));
        } else if (ty == 2) {
          const double l10 = log10(Pr);
          const double xSRI = 1. / (1. + l10 * l10);
          wF = pow(lF, xSRI) * M.D(L.fo_d)[fo];
          const double e = M.D(L.fo_e)[fo];
          if (e != 0.) wF *= pow(T, e);
        }
        // CABR (KineticsMap_CHEMKIN.hpp:1613-1660): k0 (1 / (1 + Pr)) F; fall-off: k_inf (Pr / (1 + Pr)) F
        if (cabr) kMod *= (1. / (1. + Pr)) * wF;
        else kMod *= kInf * (Pr / (1. + Pr)) * wF / kArr;
      }
      if (L.n_xfo > 0) {     // extended fall-off (KineticsMap_CHEMKIN.hpp:1672-1681)
        const int xs = M.I(L.xfo_slot)[j];
        if (xs >= 0) {
          kArr = xfo_k(M, L, xs, T, cTotSum, [&](int k) { return W.C[k]; });
          kMod = kArr;
        }
      }
      double fwd = 1.;
      for (int q = op[j]; q < op[j + 1]; ++q) fwd *= conc_factor_k(onu[q], W.C[osp[q]]);
      double net = fwd;
      const int kind = rk[j];
      if (kind != 0) {
        double rv = 1.;
        for (int q = pp[j]; q < pp[j + 1]; ++q) rv *= conc_factor_k(pnu[q], W.C[psp[q]]);
        if (kind == 1) rv *= ukeq[j];
        else rv *= ukeq[j] / kArr;
        net -= rv;
      }
      double r = net * kMod;
      if constexpr (kDrg) {
        if (W.DROP[j]) r = 0.;   // DRG-reduced system: dropped reactions (chemistry_DRG.H)
      }
      W.NET[j] = r;
    }
  }
  __syncthreads();
  double Rl = 0.;
  if (tid < NC) {
    const int* fp = M.I(L.fr_ptr);
    const int* fr = M.I(L.fr_rxn);
    const double* fc = M.D(L.fr_coef);
    for (int q = fp[tid]; q < fp[tid + 1]; ++q) {
      const double c = fc[q];
      Rl += contrib_k(c < 0. ? -c : c, W.NET[fr[q]]) * (c < 0. ? -1. : 1.);
    }
  }
  double dyl = tid < NC ? mwl * Rl / rho : 0.;
  double QR = W.slot[2];
  if (energy) {
    double cpl = 0.;
    if (tid < NC) {
      const double* A = T > TM[tid] ? M.D(L.cp_ht) + 5 * tid : M.D(L.cp_lt) + 5 * tid;
      cpl = A[0] + T * A[1] + T2 * A[2] + T3 * A[3] + T4 * A[4];
    }
    const double cpm = bsum<BT>(cpl * xl, W.red) * kRgas;
    const double d = bsum<BT>(Rl * hl, W.red);
    QR = -d * kRgas * T;
    if (cv) {
      const double CvMixMass = (cpm - kRgas) / MWmix;
      const double sumR = bsum<BT>(Rl, W.red);
      if (tid == NC) dyl = (QR + kRgas * T * sumR) / (rho0 * CvMixMass);
    } else {
      const double CpMixMass = cpm / MWmix;
      if (tid == NC) dyl = QR / (rho * CpMixMass);
    }
  } else if (tid == NC) {
    dyl = 0.;
  }
  __syncthreads();
  if (tid == 0) W.slot[2] = QR;
  __syncthreads();
  return dyl;
}

// y = A x for a column-major matrix with BT rows (leading dimension BT) and n columns; x: n doubles in
// shared memory.  Thread t reads rows 4 (t mod BT/4) .. +3 of a quarter of the columns with 16-byte
// loads (four independent streams per row quad, so that many loads are in flight); the quarters are
// summed through part (4 BT doubles, shared).  Returns y_tid.  All BT threads call it.
template <int BT, typename T>
__device__ __forceinline__ double gemv_block(const T* __restrict__ A, int n, const double* xs, double* part) {
  const int tid = threadIdx.x;
  constexpr int RQ = BT / 4;
  const int q = tid % RQ, sl = tid / RQ;
  const int js = (n * sl) >> 2, je = (n * (sl + 1)) >> 2;
  double a0 = 0., a1 = 0., a2 = 0., a3 = 0.;
  if constexpr (sizeof(T) == 4) {
    const float4* A4 = reinterpret_cast<const float4*>(A);
#pragma unroll 8
    for (int j = js; j < je; ++j) {
      const float4 v = A4[(long)j * RQ + q];
      const double xj = xs[j];
      a0 += (double)v.x * xj;
      a1 += (double)v.y * xj;
      a2 += (double)v.z * xj;
      a3 += (double)v.w * xj;
    }
  } else {
    const double2* A2 = reinterpret_cast<const double2*>(A);
#pragma unroll 4
    for (int j = js; j < je; ++j) {
      const double2 v0 = A2[(long)j * (BT / 2) + 2 * q];
      const double2 v1 = A2[(long)j * (BT / 2) + 2 * q + 1];
      const double xj = xs[j];
      a0 += v0.x * xj;
      a1 += v0.y * xj;
      a2 += v1.x * xj;
      a3 += v1.y * xj;
    }
  }
  double* pp = part + sl * BT + 4 * q;
  pp[0] = a0;
  pp[1] = a1;
  pp[2] = a2;
  pp[3] = a3;
  __syncthreads();
  const double y = (part[tid] + part[BT + tid]) + (part[2 * BT + tid] + part[3 * BT + tid]);
  __syncthreads();
  return y;
}

// ---------------------------------------------------------------------------
// Gear / multivalue BDF integrator for one block (one cell).
// ---------------------------------------------------------------------------
// DRG: the DRG-reduced system (chemistry_DRG.H) instead of the full reactor (FP64 factors only).
template <int BT, bool TC = false, bool DRG = false>
struct GearBlock {
  enum { H_DEC, H_CONST, H_INC };
  enum { O_DEC, O_CONST, O_INC };
  enum { JAC_CHANGE, JAC_MODIFIED };
  enum { M_TO_FACT, M_FACT };
  enum { CONV_FAIL, CONV_OK };

  const MechLayout* L;
  MechView M;
  BlockShared W;
  double* J;      // column-major, leading dimension jld, global
  int jld;
  double* G;      // [n][n] factors, global (FP64 form)
  // mixed-precision form (TC): the tensor-core inverse's shared memory, TMEM and barrier parity
  tc::Smem TS;
  uint32_t tmem;
  uint32_t tc_phase;
  bool tc_failed;
  double tc_hr0;    // hr0 of the matrix the current inverse belongs to
  bool tc_fp64;     // the refinement stalled on this matrix: it was refactorised by the FP64 LU
  bool tc_sticky;   // ... and the cell's later matrices go to the FP64 LU directly
  // more than 128 components (TCL): the inverse in global memory (lsg_tc.cuh gj_inverse_large), its
  // pivots in shared memory; part/ysm: the solves' partial sums (shared)
  static constexpr bool TCL = TC && BT > 128;
  float* RL;
  tc::SmemL TL;
  double* part;
  double* ysm;
  double* karr;
  double* ukeq;
  double* kinf;
  double* logf;
  double P0;
  double rho0;   // > 0: constant-volume reactor of this density
  int energy;
  int tid, ne;
  bool active;
  double b, deltab, f, va, vb, y, y0, eps, minv, maxv;
  double alfa2_4, alfa2_5;
  __device__ __forceinline__ double alfa2(unsigned k) const { return k == 4 ? alfa2_4 : (k == 5 ? alfa2_5 : .8); }
  double abs_tol, rel_tol;
  unsigned maximum_order, max_number_steps;
  double t, t0, tOut, tInMeshPoint, tStabilize;
  double hNordsieck, hScaleMax, h, hNextStep, hScale;
  bool fixedOrderMin;
  unsigned iterConstSteps, iterMinimumOrder;
  unsigned p, iterOrder, orderInNextStep, maxIterationsJacobian;
  int odeHStatus, odeOrderStatus, status, factorizationStatus, jacobianStatus, convergenceStatus;
  unsigned numberOfSteps, iterConvergence, iterConvergenceRate, iterConvergenceFailure, iterErrorFailure;
  unsigned numberOfConvergenceFailuresForOrderMax, stepOfLastJacobian;
  long long cnt[NCNT];
  // DRG-reduced system (BatchReactorHomogeneousConstantPressure.H:253-320): thread l < drg_ni owns species
  // drg_sp (the l-th important one), thread drg_ni owns T; as a thread of the full layout (species tid),
  // drg_pos is that species' reduced index or -1, drg_omega its fixed mass fraction.
  bool unconstrained = false;   // no minimum/maximum constraints: KernelDense's unconstrained increments
  int drg_ni = 0, drg_sp = 0, drg_pos = -1, drg_nc = 0;
  double drg_omega = 0.;

  __device__ __forceinline__ double& Z(int i) { return W.Z[i * BT + tid]; }
  __device__ __forceinline__ double& V(int i) { return W.V[i * BT + tid]; }

  // f(y) of the system being integrated: the full reactor, or the DRG-reduced one evaluated through the
  // full layout (kept species fixed, dropped reactions at zero rate) and gathered back
  __device__ double eval(double yl) {
    if constexpr (!DRG) {
      const double T = bcast(yl, ne - 1, W.slot);
      return rhs_block<BT>(*L, M, W, karr, ukeq, kinf, logf, yl, T, P0, energy, rho0);
    } else {
      __syncthreads();
      W.DX[tid] = yl;   // reduced layout
      __syncthreads();
      const double T = W.DX[drg_ni];
      const double yf = tid < drg_nc ? (drg_pos >= 0 ? W.DX[drg_pos] : drg_omega) : T;
      const double df = rhs_block<BT, true>(*L, M, W, karr, ukeq, kinf, logf, yf, T, P0, energy, rho0);
      __syncthreads();
      W.DX[tid] = df;   // full layout
      __syncthreads();
      return W.DX[drg_sp];
    }
  }

  __device__ double rhs(double yl) {
    ++cnt[CNT_RHS];
    return eval(yl);
  }

  __device__ double error_control(double w) {   // OpenSMOKEUtilities.hpp:689-701
    const double c = active ? w * eps : 0.;
    return sqrt(bsum<BT>(c * c, W.red) / double(ne));
  }

  __device__ __forceinline__ void check_constraints(double& yl) {
    if (active) {
      if (yl < minv) yl = minv;
      if (yl > maxv) yl = maxv;
    }
  }

  __device__ __forceinline__ void one_over_epsilon(double w) {
    if (active) eps = 1. / (abs_tol + rel_tol * fabs(w));
  }

  // KernelDense::NumericalJacobian, constrained branch (KernelDense.hpp:111-193)
  __device__ void numerical_jacobian(double yl, double fl) {
    const double ZERO_DER = sqrt(kTinyFloat);
    const double ETA2 = sqrt(kMachEpsDouble);
    const double BETA = 1.e+3 * kMachEpsDouble;
    double hf = BETA * fabs(h) * error_control(fl) * double(ne);
    if (hf < 1.e-10) hf = 1.;
    const int n = ne;
    for (int j = 0; j < n; ++j) {
      const double yh = bcast(yl, j, W.slot);
      const double ej = bcast(eps, j, W.slot);
      const double mxj = bcast(maxv, j, W.slot);
      double hJ;
      if (DRG && unconstrained) {   // KernelDense.hpp:111-193 without maximum constraints
        hJ = ETA2 * fabs(fmax(yh, 1. / ej));
        hJ = fmax(hJ, hf / ej);
        hJ = fmax(hJ, ZERO_DER);
        hJ = fmin(hJ, 0.001 + 0.001 * fabs(yh));
      } else {
        const double a = fabs(yh), bb = fabs(1. / ej);
        hJ = ETA2 * (a > bb ? a : bb);
        hJ = fmax(hJ, hf / ej);
        hJ = fmax(hJ, ZERO_DER);
        if (yh + hJ > mxj) hJ = -hJ;
      }
      double yp = yl;
      if (tid == j) yp += hJ;
      const double aux = eval(yp);
      ++cnt[CNT_JAC_RHS];
      const double hInv = 1. / hJ;
      if (active) J[(long)j * jld + tid] = hInv * (aux - fl);
    }
    __syncthreads();
  }

  // G = I - hr0 J; partial-pivot LU (largest magnitude, first occurrence).
  // Column storage: G(i, j) at G[j * n + i].
  __device__ void build_and_factorize(double hr0) {
    if constexpr (TC) {
      if (tc_sticky) {   // this cell's matrices defeated the FP32 inverse before
        build_and_factorize_fp64(hr0);
        tc_hr0 = hr0;
        tc_fp64 = true;
        return;
      }
      // G^-1 in FP32 by the tensor-core Gauss-Jordan inverse (lsg_tc.cuh)
      if constexpr (TCL) {
        if (!tc::gj_inverse_large<BT / 128>(J, jld, ne, hr0, RL, TL, tmem, &tc_phase)) tc_failed = true;
      } else {
        if (!tc::gj_inverse(J, ne, hr0, TS, tmem, &tc_phase)) tc_failed = true;
      }
      tc_hr0 = hr0;
      tc_fp64 = false;
      ++cnt[CNT_FACT];
    } else {
      build_and_factorize_fp64(hr0);
    }
  }

  __device__ void build_and_factorize_fp64(double hr0) {
    const int n = ne;
    for (long e = tid; e < (long)n * n; e += BT) {
      const int j = (int)(e / n), i = (int)(e % n);
      double g = J[(long)j * jld + i];
      g *= -hr0;
      if (i == j) g += 1.;
      G[e] = g;
    }
    __syncthreads();
    for (int k = 0; k < n; ++k) {
      // pivot search over rows k..n-1 of column k, ties -> lowest row
      double best = (tid >= k && tid < n) ? fabs(G[(long)k * n + tid]) : -1.;
      int row = tid;
      for (int off = 16; off > 0; off >>= 1) {
        const double ob = __shfl_xor_sync(kFull, best, off);
        const int orow = __shfl_xor_sync(kFull, row, off);
        if (ob > best || (ob == best && orow < row)) { best = ob; row = orow; }
      }
      if ((tid & 31) == 0) { W.red[tid >> 5] = best; W.ival[tid >> 5] = row; }
      __syncthreads();
      if (tid < 32) {
        double bv = tid < BT / 32 ? W.red[tid] : -2.;
        int br = tid < BT / 32 ? W.ival[tid] : (1 << 30);
        for (int off = 16; off > 0; off >>= 1) {
          const double ob = __shfl_xor_sync(kFull, bv, off);
          const int orow = __shfl_xor_sync(kFull, br, off);
          if (ob > bv || (ob == bv && orow < br)) { bv = ob; br = orow; }
        }
        if (tid == 0) W.ival[BT / 32] = (br >= k && br < n) ? br : k;
      }
      __syncthreads();
      const int pr = W.ival[BT / 32];
      if (tid == 0) W.PIV[k] = pr;
      // swap rows k and pr and stage the new row k (the pivot row) in shared memory (W.X is free here)
      for (int j = tid; j < n; j += BT) {
        double gk = G[(long)j * n + k];
        if (pr != k) {
          const double gp = G[(long)j * n + pr];
          G[(long)j * n + pr] = gk;
          G[(long)j * n + k] = gp;
          gk = gp;
        }
        W.X[j] = gk;
      }
      __syncthreads();
      // thread i > k owns row i: its multiplier, then the row's rank-1 update (each element is updated
      // once per k, so the result does not depend on this loop order)
      if (tid > k && tid < n) {
        const double d = W.X[k];
        double l = G[(long)k * n + tid];
        if (d != 0.) l /= d;
        G[(long)k * n + tid] = l;
        // G lives in global memory: the row's elements are loaded eight at a time before any of them is
        // written back, so their L2 latencies overlap (a store may alias a later load, so the compiler
        // cannot reorder them itself)
        double* Gr = G + tid;
        int j = k + 1;
        for (; j + 8 <= n; j += 8) {
          double g[8];
#pragma unroll
          for (int q = 0; q < 8; ++q) g[q] = Gr[(long)(j + q) * n];
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            g[q] -= l * W.X[j + q];
            Gr[(long)(j + q) * n] = g[q];
          }
        }
        for (; j < n; ++j) Gr[(long)j * n] -= l * W.X[j];
      }
      __syncthreads();
    }
    // the row interchanges composed, for the solves: apply PIV[0..n-1] in order to the identity
    if (tid == 0) {
      for (int i = 0; i < n; ++i) W.PERM[i] = i;
      for (int k = 0; k < n; ++k) {
        const int pk = W.PIV[k];
        if (pk != k) {
          const int t2 = W.PERM[k];
          W.PERM[k] = W.PERM[pk];
          W.PERM[pk] = t2;
        }
      }
    }
    __syncthreads();
    ++cnt[CNT_FACT];
  }

  // KernelDense::SolveLinearSystem with the factors of build_and_factorize:
  // row interchanges, then column-oriented forward and back substitution.
  // x = X r with the FP32 inverse X (column-major in shared memory), accumulated in FP64
  __device__ double apply_inverse(double rl) {
    const int n = ne;
    if constexpr (TCL) {
      // x_a = y_{p_a}, y = R r~, r~_s = r_{p_s} (gj_inverse_large); after a failed inverse the pivots are
      // incomplete: the solve is discarded then, but stays in bounds
      W.X[tid] = 0.;
      __syncthreads();
      const int sl = TL.colof[tid];
      if (tid < n && sl >= 0 && sl < n) W.X[sl] = rl;
      __syncthreads();
      const double y = gemv_block<BT, float>(RL, n, W.X, part);
      ysm[tid] = y;
      __syncthreads();
      const double x = tid < n ? ysm[TL.piv[tid]] : 0.;
      __syncthreads();
      return x;
    }
    W.X[tid] = tid < n ? rl : 0.;
    __syncthreads();
    double x = 0.;
    if (tid < n) {
      const float* RT = TS.op;
#pragma unroll 4
      for (int j = 0; j < n; ++j) x += (double)RT[j * tc::kRows + tid] * W.X[j];
    }
    __syncthreads();
    return x;
  }

  // (G x)_tid = x_tid - hr0 (J x)_tid in FP64 with the FP64 Jacobian (column-major in global memory)
  __device__ double apply_g(double xl, double hr0) {
    return xl - hr0 * jacobian_times(xl);
  }

  // (J x)_tid, FP64
  __device__ double jacobian_times(double xl) {
    const int n = ne;
    W.X[tid] = tid < n ? xl : 0.;
    __syncthreads();
    if constexpr (TCL) return gemv_block<BT, double>(J, n, W.X, part);
    double s0 = 0.;   // JacobianTimesVector (MethodGear.hpp:438) in column order
    if (tid < n) {
#pragma unroll 8
      for (int j = 0; j < n; ++j) s0 += J[(long)j * jld + tid] * W.X[j];
    }
    __syncthreads();
    return s0;
  }

  // Mixed-precision solve: x = X r, then refinement sweeps x += X (r - G x) on the FP64 residual until
  // the weighted RMS of a correction is below kBlkRefineTol (the Newton test compares such norms with 1), at
  // most kBlkRefineMax sweeps.  Each sweep must at least halve the weighted norm of the residual (the
  // first against r): otherwise X is no usable inverse of G (FP32 cannot hold this matrix's conditioning,
  // and a correction X res can be small while the residual is not), G is refactorised by the FP64 LU, and
  // the cell's remaining factorisations stay FP64 (tc_sticky).
  __device__ double solve(double xl) {
    if constexpr (TC) {
      if (!tc_fp64) {
        double x = apply_inverse(xl);
        double prev = error_control(xl);
        bool converged = false;
        for (int s = 0; s < kBlkRefineMax; ++s) {
          const double res = xl - apply_g(x, tc_hr0);
          const double rr = error_control(res);
          if (!(rr <= 0.5 * prev || rr == 0.)) break;   // (a NaN residual breaks too)
          prev = rr;
          const double d = apply_inverse(res);
          x += d;
          if (error_control(d) <= kBlkRefineTol) { converged = true; break; }
        }
        if (converged) {
          ++cnt[CNT_SOLVE];
          return x;
        }
        build_and_factorize_fp64(tc_hr0);   // the same matrix: not a factorisation of the method
        --cnt[CNT_FACT];
        tc_fp64 = true;
        tc_sticky = true;
      }
      return solve_fp64(xl);
    } else {
      return solve_fp64(xl);
    }
  }

  __device__ double solve_fp64(double xl) {
    const int n = ne;
    W.X[tid] = tid < n ? xl : 0.;
    __syncthreads();
    const double xp = tid < n ? W.X[W.PERM[tid]] : 0.;   // the row interchanges of the factorisation
    __syncthreads();
    W.X[tid] = xp;
    __syncthreads();
    // Substitution in panels of 32 columns.  Warp 0 solves a panel's diagonal
    // block with shuffles, the rows below (above, going back) then apply the
    // panel's columns; two block barriers per panel instead of one per column.
    // Every row still applies its updates one column at a time in the
    // column-oriented order (forward: j ascending; back: j descending, then
    // the division by its pivot), so the result is the same to the last bit.
    double x = W.X[tid];
    for (int j0 = 0; j0 < n; j0 += 32) {
      const int j1 = min(j0 + 32, n);
      if (tid >= j0 && tid < j1) W.X[tid] = x;
      __syncthreads();
      if (tid < 32) {
        const int r = j0 + tid;
        double xr = r < j1 ? W.X[r] : 0.;
        // the diagonal block's row r, loaded 16 columns ahead so the global-memory latencies overlap
#pragma unroll
        for (int c = 0; c < 32; c += 16) {
          double g[16];
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const int j = j0 + c + q;
            g[q] = (r < j1 && j < j1) ? G[(long)j * n + r] : 0.;
          }
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const int j = j0 + c + q;
            if (j < j1) {   // the same in every lane
              const double xj = __shfl_sync(kFull, xr, c + q);
              if (r > j && r < j1) xr -= g[q] * xj;
            }
          }
        }
        if (r < j1) W.X[r] = xr;
      }
      __syncthreads();
      if (tid >= j1 && tid < n) {
        int j = j0;
        for (; j + 8 <= j1; j += 8) {
          double g[8];
#pragma unroll
          for (int q = 0; q < 8; ++q) g[q] = G[(long)(j + q) * n + tid];
#pragma unroll
          for (int q = 0; q < 8; ++q) x -= g[q] * W.X[j + q];
        }
        for (; j < j1; ++j) x -= G[(long)j * n + tid] * W.X[j];
      } else if (tid >= j0 && tid < j1) {
        x = W.X[tid];
      }
    }
    for (int j1 = n; j1 > 0; j1 -= 32) {
      const int j0 = max(j1 - 32, 0);
      if (tid >= j0 && tid < j1) W.X[tid] = x;
      __syncthreads();
      if (tid < 32) {
        const int r = j0 + tid;
        double xr = r < j1 ? W.X[r] : 0.;
#pragma unroll
        for (int c = 0; c < 32; c += 16) {
          double g[16];
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const int j = j1 - 1 - c - q;
            g[q] = (r < j1 && j >= j0) ? G[(long)j * n + r] : 0.;
          }
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const int j = j1 - 1 - c - q;
            if (j >= j0) {   // the same in every lane
              if (r == j) xr /= g[q];
              const double xj = __shfl_sync(kFull, xr, j - j0);
              if (r < j) xr -= g[q] * xj;
            }
          }
        }
        if (r < j1) W.X[r] = xr;
      }
      __syncthreads();
      if (tid < j0) {
        int j = j1 - 1;
        for (; j - 8 >= j0 - 1; j -= 8) {
          double g[8];
#pragma unroll
          for (int q = 0; q < 8; ++q) g[q] = G[(long)(j - q) * n + tid];
#pragma unroll
          for (int q = 0; q < 8; ++q) x -= g[q] * W.X[j - q];
        }
        for (; j >= j0; --j) x -= G[(long)j * n + tid] * W.X[j];
      } else if (tid < j1) {
        x = W.X[tid];
      }
    }
    __syncthreads();
    ++cnt[CNT_SOLVE];
    return tid < n ? x : 0.;
  }

  __device__ void set_initial_conditions(double tstart, double y0l) {
    tOut = t = t0 = tInMeshPoint = tStabilize = tstart;
    p = 1; iterOrder = 0; orderInNextStep = 1;
    maxIterationsJacobian = 20 + 5 * (unsigned)(ne - 3);
    if (maxIterationsJacobian > 50u && ne < 80) maxIterationsJacobian = 50u;
    odeHStatus = H_CONST; odeOrderStatus = O_CONST; status = 1;
    factorizationStatus = M_TO_FACT; jacobianStatus = JAC_CHANGE; convergenceStatus = CONV_OK;
    h = 0.; hNextStep = 0.; hScale = 0.;
    numberOfSteps = 0; numberOfConvergenceFailuresForOrderMax = 0;
    iterConvergence = 0; iterConvergenceRate = 0; iterConvergenceFailure = 0; iterErrorFailure = 0;
    stepOfLastJacobian = 0;
    y0 = y0l;
    hNordsieck = 0.; hScaleMax = 1000.;
    fixedOrderMin = false; iterConstSteps = 0; iterMinimumOrder = 0;
    for (int k = 0; k < NCNT; ++k) cnt[k] = 0;
    f = rhs(y0);
  }

  __device__ unsigned find_correction() {   // MethodGear.hpp:195-341
    vb = active ? V(0) : 0.;
    check_constraints(vb);
    f = rhs(vb);
    if (numberOfSteps >= stepOfLastJacobian + maxIterationsJacobian) jacobianStatus = JAC_CHANGE;
    if (jacobianStatus == JAC_CHANGE) {
      stepOfLastJacobian = numberOfSteps;
      jacobianStatus = JAC_MODIFIED;
      numerical_jacobian(vb, f);
      ++cnt[CNT_JAC];
      factorizationStatus = M_TO_FACT;
    }
    const double r0 = c_gear_k.r[0][p - 1];
    const double hr0 = h * r0;
    if (factorizationStatus == M_FACT && iterOrder == 0) factorizationStatus = M_TO_FACT;
    if (factorizationStatus == M_TO_FACT) {
      build_and_factorize(hr0);
      factorizationStatus = M_FACT;
    }
    deltab = f * h;
    deltab -= active ? V(1) : 0.;
    deltab = solve(deltab);
    b = deltab;
    double oldCC = 0.;
    for (unsigned k = 1; k <= 4; ++k) {
      const double cc = r0 * error_control(deltab);
      if (cc < 1.) { convergenceStatus = CONV_OK; return k; }
      if (k > 1 && cc > 2. * oldCC) { convergenceStatus = CONV_FAIL; return k; }
      oldCC = cc;
      va = b * r0;
      va += active ? V(0) : 0.;
      if (active) {
        if (va < minv) { va = minv; b = (minv - Z(0)) / r0; }
        if (va > maxv) { va = maxv; b = (maxv - Z(0)) / r0; }
      }
      f = rhs(va);
      deltab = f * h;
      deltab -= active ? V(1) : 0.;
      deltab -= b;
      deltab = solve(deltab);
      b += deltab;
    }
    convergenceStatus = CONV_FAIL;
    return 4;
  }

  __device__ void convergence_failure_recovery() {   // MethodGear.hpp:343-423
    hScale = 0.25;
    if (numberOfSteps < 10) hScale = 0.1;
    hScale = fmax(hScale, 0. / fabs(h));
    odeHStatus = H_DEC;
    if (p > 1u) { p -= 1; odeOrderStatus = O_DEC; }
    alfa2_4 -= 0.01;
    alfa2_5 -= 0.02;
    if (alfa2_4 < 0.) { alfa2_4 = 0.; maximum_order = 3; if (p > 3) { p = 3; odeOrderStatus = O_DEC; } }
    if (alfa2_5 < 0.) { alfa2_5 = 0.; maximum_order = 4; if (p > 4) { p = 4; odeOrderStatus = O_DEC; } }
    if (numberOfSteps > 5) {
      numberOfConvergenceFailuresForOrderMax++;
      if (numberOfConvergenceFailuresForOrderMax % 5 == 0 && p != 1u) { p = 1; odeOrderStatus = O_DEC; }
      if (numberOfConvergenceFailuresForOrderMax % 10 == 0 && tStabilize != tInMeshPoint) {
        va = rhs(active ? Z(0) : 0.);
        if (active) Z(1) = va * h;
        tStabilize = tInMeshPoint;
      }
    }
    if (numberOfSteps > stepOfLastJacobian + 5u) jacobianStatus = JAC_CHANGE;
    if (numberOfSteps != stepOfLastJacobian && iterConvergenceFailure == 50u) jacobianStatus = JAC_CHANGE;
    hNextStep *= hScale;
  }

  __device__ void convergence_rate() {   // MethodGear.hpp:425-516
    if (iterErrorFailure > 0 || iterConvergenceFailure > 0) iterConvergenceRate = 0;
    if (iterConvergence <= 1) return;
    const double s = jacobian_times(active ? V(0) - Z(0) : 0.);
    va = active ? s : 0.;
    va *= h;
    va += active ? Z(1) : 0.;
    va = (active ? V(1) : 0.) - va;
    const double normd = bsum<BT>(active ? fabs(va) : 0., W.red);
    const double normf = bsum<BT>(active ? fabs(V(1)) : 0., W.red);
    if (normd > 3. * normf + .1 && iterConvergence > 2) {
      if (numberOfSteps > stepOfLastJacobian + 5u) jacobianStatus = JAC_CHANGE;
      hScale = 0.5; odeHStatus = H_DEC; hNextStep = h * hScale;
      if (p > 1) { orderInNextStep = p - 1; odeOrderStatus = O_DEC; }
      iterConvergenceRate = 0; iterConvergenceFailure = 1;
      return;
    }
    if (normd > normf + 0.1) {
      iterConvergenceRate++;
      if (iterConvergenceRate >= 5) {
        hScale = 0.8; odeHStatus = H_DEC; hNextStep = h * hScale;
        iterConvergenceRate = 0; iterConvergenceFailure = 1;
      }
      if (numberOfSteps > stepOfLastJacobian + 5u && iterConvergence > 2) {
        jacobianStatus = JAC_CHANGE;
        iterConvergenceRate = 0; iterConvergenceFailure = 1;
      }
    }
  }

  __device__ void multi_value_step() {   // MultiValueSolver.hpp:1212-1327
    if (active) {
      for (unsigned i = 0; i <= p; ++i) V(i) = Z(i);
      for (int i = 0; i < int(p); ++i)
        for (int j = int(p) - 1; j >= i; --j) V(j) += V(j + 1);
      if (V(0) < minv && fabs(V(0) - minv) * eps < double(ne)) {
        V(0) = minv; V(1) = minv - Z(0);
        for (unsigned i = 2; i <= p; ++i) V(i) = 0.;
      }
      if (V(0) > maxv && fabs(V(0) - maxv) * eps < double(ne)) {
        V(0) = maxv; V(1) = maxv - Z(0);
        for (unsigned i = 2; i <= p; ++i) V(i) = 0.;
      }
    }
    iterConvergence = find_correction();
    if (convergenceStatus == CONV_FAIL) return;
    const double r0 = c_gear_k.r[0][p - 1];
    if (active) {
      va = b * r0;
      if (V(0) + va < minv) { b = minv - Z(0) - V(1); V(0) = minv - va; if (V(0) < minv) V(0) = minv; }
      if (V(0) + va > maxv) { b = maxv - Z(0) - V(1); V(0) = maxv - va; if (V(0) > maxv) V(0) = maxv; }
      V(0) += va;
      V(1) += b;
      for (unsigned i = 2; i <= p; ++i) V(i) += b * c_gear_k.r[i][p - 1];
      V(p + 1) = (V(p) - Z(p)) / (double(p) + 1.);
      if (iterOrder >= p) V(p + 2) = (V(p + 1) - Z(p + 1)) / (double(p) + 2.);
    }
  }

  __device__ void new_order_new_h() {   // MultiValueSolver.hpp:1042-1210
    double hMinus = 0., hCur = 0., hPlus = 0., alfa1 = 0., alfa3 = 0.;
    if (p > 1u && odeOrderStatus != O_INC) {
      hMinus = c_gear_k.Ep[p - 1] * error_control(active ? V(p) : 0.) + kMachEpsFloat;
      hMinus = 1. / hMinus;
      alfa1 = alfa2(p - 1) - .05;
      hMinus = alfa1 * pow(hMinus, 1. / double(p));
    }
    hCur = c_gear_k.Ep[p] * error_control(active ? V(p + 1) : 0.) + kMachEpsFloat;
    hCur = 1. / hCur;
    hCur = alfa2(p) * pow(hCur, 1. / double(p + 1));
    if (p < maximum_order && odeOrderStatus != O_DEC) {
      hPlus = c_gear_k.Ep[p + 1] * error_control(active ? V(p + 2) : 0.) + kMachEpsFloat;
      hPlus = 1. / hPlus;
      alfa3 = alfa2(p + 1) - .25;
      hPlus = alfa3 * pow(hPlus, 1. / double(p + 2));
    }
    if (hMinus > hCur && hMinus > hPlus) {
      hScale = (.75 / alfa1) * hMinus; orderInNextStep = p - 1; odeOrderStatus = O_DEC;
    } else if (hCur > hMinus && hCur > hPlus) {
      hScale = (.75 / alfa2(p)) * hCur; orderInNextStep = p; odeOrderStatus = O_CONST;
    } else {
      hScale = (.75 / alfa3) * hPlus; orderInNextStep = p + 1; odeOrderStatus = O_INC;
    }
    if (fixedOrderMin) {
      iterMinimumOrder++;
      if (iterMinimumOrder < 2000) {
        hScale = (.75 / alfa2(p)) * hCur; orderInNextStep = p; odeOrderStatus = O_CONST;
      } else {
        fixedOrderMin = false;
      }
    }
    if (hScale < 1.2) {
      iterConstSteps++;
      hScale = 1.; odeHStatus = H_CONST; orderInNextStep = p; odeOrderStatus = O_CONST; hNextStep = h;
    } else {
      iterConstSteps = 0;
      hScale = fmin(hScale, hScaleMax);
      odeHStatus = H_INC;
      hNextStep = h * hScale;
    }
    if (iterConstSteps > 500 ||
        (numberOfSteps % 1000 == 0 && numberOfSteps != 0 && (fabs(h) < 1.e-7 || fabs(h) < 1.e-5 * t))) {
      if (p > 1u) {
        fixedOrderMin = true; iterMinimumOrder = 0;
        orderInNextStep = 1; odeOrderStatus = O_DEC;
        hScale = 0.5; hNextStep = h * hScale; odeHStatus = H_DEC;
      }
    }
  }

  __device__ void driver_step() {   // MultiValueSolver.hpp:753-1040
    iterConvergenceFailure = 0; iterErrorFailure = 0; convergenceStatus = CONV_OK;
    if (odeOrderStatus != O_CONST || odeHStatus != H_CONST) iterOrder = 0;
    p = orderInNextStep;
    odeOrderStatus = O_CONST;
    hScaleMax = 2.;
    if (numberOfSteps < 10) hScaleMax = 1000.;
    else if (numberOfSteps > 10 && numberOfSteps < 20) hScaleMax = 10.;
    for (int guard = 0; guard < 1000000; ++guard) {
      if constexpr (TC) {
        if (tc_failed) { status = -1; return; }   // an MMA did not complete: the cell stops
      }
      if (odeHStatus != H_CONST) {
        hScale = hNextStep / hNordsieck;
        double hr = 1.;
        for (unsigned i = 1; i <= p; ++i) {
          hr *= hScale;
          if (active) Z(i) *= hr;
        }
        if (active) { double z0 = Z(0); check_constraints(z0); Z(0) = z0; }
        iterOrder = 0;
        odeHStatus = H_CONST;
      }
      h = hNextStep;
      hNordsieck = hNextStep;
      t = tInMeshPoint + h;
      if (t == tInMeshPoint) { status = -6; return; }
      multi_value_step();
      if (convergenceStatus == CONV_FAIL) {
        iterConvergenceFailure++;
        ++cnt[CNT_CONVFAIL];
        if (iterConvergenceFailure >= 50u) { status = -5; return; }
        if (fabs(h) <= 0.) { status = -6; return; }
        convergence_failure_recovery();
      } else {
        double hCur = c_gear_k.Ep[p] * error_control(active ? V(p + 1) : 0.);
        if (hCur > 1.) {
          iterErrorFailure++;
          ++cnt[CNT_ERRFAIL];
          if (iterErrorFailure >= 50u) { status = -4; return; }
          if (fabs(h) <= 0.) { status = -6; return; }
          hScaleMax = 1.;
          hCur = 0.8 * pow(1. / hCur, 1. / double(p + 1));
          hScale = hCur;
          if (p > 1u) {
            double hMinus = c_gear_k.Ep[p - 1] * error_control(active ? V(p) : 0.);
            hMinus = 1. / (hMinus + kMachEpsFloat);
            hMinus = 0.8 * pow(hMinus, 1. / double(p));
            if (hMinus > hCur) { hScale = hMinus; p -= 1; odeOrderStatus = O_DEC; }
          }
          hScale = fmin(hScale, 0.5);
          hScale = fmax(hScale, 0. / fabs(h));
          hScale = fmax(hScale, 1.e-3);
          if (p == 1 && hScale < 0.1 && numberOfSteps > 10 && tInMeshPoint != tStabilize) {
            va = rhs(active ? Z(0) : 0.);
            if (active) Z(1) = va * h;
            tStabilize = tInMeshPoint;
          }
          odeHStatus = H_DEC;
          hNextStep *= hScale;
        } else {
          hNordsieck = h; hNextStep = h;
          orderInNextStep = p; odeOrderStatus = O_CONST; odeHStatus = H_CONST;
          convergence_rate();
          if (iterErrorFailure > 0 || iterConvergenceFailure > 0) {
            iterErrorFailure = 0; iterConvergenceFailure = 0;
          } else {
            iterOrder++;
            if (iterOrder > p + 1) new_order_new_h();
          }
          if (active) {
            for (unsigned i = 0; i <= p + 2; ++i) Z(i) = V(i);
            double z0 = Z(0); check_constraints(z0); Z(0) = z0;
          }
          return;
        }
      }
    }
    status = -5;
  }

  // MultiValueSolver::Solve from a fresh initial condition (:423-617); on
  // failure y holds the last accepted state.
  __device__ int solve_to(double tEnd) {
    tOut = tEnd;
    const bool illegal = active && (y0 < minv || y0 > maxv);
    if (__syncthreads_or(illegal)) { status = -9; y = y0; return status; }
    one_over_epsilon(y0);
    double lo, hi;
    if (t0 != 0.) { lo = 100. * kMachEpsDouble * fabs(t0); hi = fabs(t0); }
    else { lo = kMachEpsDouble; hi = 1.e-4; }
    double h0 = 0.5 / (error_control(f) + kMachEpsFloat);
    if (h0 < lo) h0 = lo;
    if (h0 > hi) h0 = hi;
    h0 *= fabs(tOut - t0) / (tOut - t0);
    if (active) { Z(0) = y0; Z(1) = f * h0; }
    hNordsieck = h0; hNextStep = h0;
    status = 2;
    for (unsigned k = 1; k <= max_number_steps; ++k) {
      one_over_epsilon(active ? Z(0) : 0.);
      const double tolSafe = kMachEpsDouble * error_control(active ? Z(0) : 0.);
      if (tolSafe > 1.) { status = -2; y = active ? Z(0) : 0.; return status; }
      tInMeshPoint = t;
      driver_step();
      if constexpr (TC) {
        if (tc_failed) status = -1;   // the device error flag reports it; the cell stops here
      }
      if (status <= 0) { t = tInMeshPoint; y = active ? Z(0) : 0.; return status; }
      numberOfSteps++;
      ++cnt[CNT_STEPS];
      if (tOut == t) { y = active ? Z(0) : 0.; return status; }
      if (tOut < t) {
        const double hp = (tOut - t) / hNordsieck;
        double hr = 1.;
        y = active ? Z(0) : 0.;
        if (hp != 0.) {
          for (unsigned i = 1; i <= p; ++i) {
            hr *= hp;
            if (active) y += Z(i) * hr;
          }
          check_constraints(y);
        }
        va = rhs(y);   // the reactor's QR at tOut
        return status;
      }
    }
    status = -1;
    y = active ? Z(0) : 0.;
    return status;
  }
};

}  // namespace

// ---------------------------------------------------------------------------
// Persistent block-per-cell kernel: blocks take cells from the queue.
// chemistry_DI.H:92-235: gather, clip and renormalise, integrate, renormalise, scatter.
// ---------------------------------------------------------------------------
template <int BT, bool TC>
__global__ void __launch_bounds__(BT, TC ? (BT == 128 ? 2 : 1) : (BT == 128 ? 4 : (BT == 256 ? 2 : 1)))
    block_kernel(MechLayout L, const unsigned char* __restrict__ mech_gmem, StepOptions o, StepArgs a,
                 double* __restrict__ ws_all, int* queue, int* err) {
  constexpr bool TCL = TC && BT > 128;
  extern __shared__ __align__(16) unsigned char bsm[];
  __shared__ int s_cell;
  const int tid = threadIdx.x;
  const int NC = L.nc, ne = NC + 1;
  const size_t wsd = block_ws_doubles(L);
  double* ws = ws_all + (size_t)blockIdx.x * wsd;
  BlockShared W;
  // global work space: the FP64 layout, or (TCL) J with leading dimension BT, G, the FP32 inverse, Z, V
  double* Jp = ws;
  int jld = ne;
  double* Gp = ws + (size_t)ne * ne;
  double* karr = ws + 2 * (size_t)ne * ne;
  float* RL = nullptr;
  tc::SmemL TL{};
  double* part = nullptr;
  double* ysm = nullptr;
  uint32_t* tslot = nullptr;
  if constexpr (TCL) {
    jld = BT;
    Gp = ws + (size_t)BT * BT;
    RL = (float*)(Gp + round32((size_t)ne * ne));
    double* zv = (double*)(RL + (size_t)BT * BT);
    W.Z = zv;
    W.V = zv + 8 * BT;
    karr = zv + 16 * BT;
    double* p = (double*)bsm;
    W.X = p; p += BT;
    W.red = p; p += BT / 32 + 1;
    W.slot = p; p += 4;
    int* ip = (int*)p;
    W.PIV = ip; ip += BT;
    W.ival = ip; ip += BT / 32 + 1;
    W.PERM = ip; ip += BT;
    TL.piv = ip; ip += BT;
    TL.colof = ip; ip += BT;
    tslot = (uint32_t*)ip; ip += 4;
    TL.mbar = (unsigned long long*)(((uintptr_t)ip + 7) & ~(uintptr_t)7);
    const uint32_t s0 = tc::smem_addr(bsm);
    const uint32_t base = ((s0 + (uint32_t)tcl_head_bytes<BT>() + 1023u) & ~1023u) - s0;
    unsigned char* un = bsm + base;
    double* d = (double*)un;
    W.C = d; d += NC;
    W.H = d; d += NC;
    W.S = d; d += NC;
    W.NET = d;
    TL.A = (float*)un;
    TL.B = TL.A + 2 * (BT / 128) * tc::kOperandFloats;
    float* f = TL.B + 2 * tc::kOperandFloats;
    TL.red = f; f += 32;
    TL.redi = (int*)f; f += 32;
    TL.prow = f;
    part = (double*)un;
    ysm = part + 4 * BT;
  } else {
    double* p = (double*)bsm;
    W.Z = p; p += 8 * BT;
    W.V = p; p += 8 * BT;
    W.C = p; p += NC;
    W.H = p; p += NC;
    W.S = p; p += NC;
    W.NET = p; p += L.nr;
    W.X = p; p += BT;
    W.red = p; p += BT / 32 + 1;
    W.slot = p; p += 4;
    W.PIV = (int*)p;
    W.ival = W.PIV + BT;
    W.PERM = W.ival + BT / 32 + 1;
  }
  // mixed-precision form: the tensor-core inverse's operands after the FP64 work space, 1024-byte aligned,
  // then its small arrays; TMEM (256 columns) for the block's lifetime
  tc::Smem TS{};
  uint32_t tmem = 0;
  if constexpr (TCL) {
    if (tid < 32) tc::tmem_alloc(tslot, BT);
    if (tid == 0) tc::mbar_init(TL.mbar, 1);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    tmem = *tslot;
  } else if constexpr (TC) {
    const uint32_t s0 = tc::smem_addr(bsm);
    const uint32_t base = ((s0 + (uint32_t)block_shared_bytes<BT>(L) + 1023u) & ~1023u) - s0;   // 1024-byte aligned
    unsigned char* q = bsm + base;
    TS.op = (float*)q; q += 4 * tc::kOperandFloats * sizeof(float);
    TS.mbar = (unsigned long long*)q; q += 16;
    TS.tmem_slot = (uint32_t*)q; q += 16;
    TS.red = (float*)q; q += 8 * sizeof(float);
    TS.redi = (int*)q; q += 8 * sizeof(int);
    TS.prow = (float*)q; q += 4 * tc::kPanel * sizeof(float);
    TS.pivot_of_row = (int*)q;
    if (tid < 32) tc::tmem_alloc(TS.tmem_slot, tc::kCols);
    if (tid == 0) tc::mbar_init(TS.mbar, 1);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    tmem = *TS.tmem_slot;
  }
  uint32_t tc_phase = 0;
  bool tc_failed = false;
  const MechView M{(const double*)mech_gmem, (const int*)(mech_gmem + (size_t)L.n_double * sizeof(double))};
  for (;;) {
    __syncthreads();
    if (tid == 0) s_cell = atomicAdd(queue, 1);
    __syncthreads();
    const long cell = s_cell;
    if (cell >= a.ncells || tc_failed) break;
    double yl = 0.;
    if (tid < NC) yl = a.Y[(size_t)tid * a.ld + cell];
    const double Tc = a.T[cell];
    if (tid == NC) yl = Tc;
    double yf = yl;
    int st = 0;
    long long nsteps = 0;
    double Q = 0.;
    if (Tc > o.tmin_chem) {
      double y0 = yl;
      if (tid < NC && y0 < 0.) y0 = 0.;
      const double sum = bsum<BT>(tid < NC ? y0 : 0., W.red);
      if (tid < NC) y0 /= sum;
      if (tid == 0) { W.slot[1] = 0.; W.slot[2] = 0.; }
      __syncthreads();
      GearBlock<BT, TC> g;
      g.TS = TS;
      g.tmem = tmem;
      g.tc_phase = tc_phase;
      g.tc_failed = false;
      g.tc_hr0 = 0.;
      g.tc_fp64 = false;
      g.tc_sticky = false;
      g.L = &L;
      g.M = M;
      g.W = W;
      g.J = Jp;
      g.jld = jld;
      g.G = Gp;
      g.RL = RL;
      g.TL = TL;
      g.part = part;
      g.ysm = ysm;
      g.karr = karr;
      g.ukeq = g.karr + L.nr;
      g.kinf = g.ukeq + L.nr;
      g.logf = g.kinf + (L.n_fo > 0 ? L.n_fo : 1);
      g.P0 = a.p;
      g.rho0 = a.rho ? a.rho[cell] : 0.;
      g.energy = o.energy;
      g.tid = tid;
      g.ne = ne;
      g.active = tid < ne;
      g.alfa2_4 = o.alfa2_4;
      g.alfa2_5 = o.alfa2_5;
      g.maximum_order = (unsigned)o.maximum_order;
      g.max_number_steps = (unsigned)o.max_steps;
      g.abs_tol = o.atol;
      g.rel_tol = o.rtol;
      g.minv = tid < NC ? 0. : o.y_min_T;
      g.maxv = tid < NC ? 1. : o.y_max_T;
      g.b = g.deltab = g.f = g.va = g.vb = g.y = 0.;
      g.eps = 0.;
      g.set_initial_conditions(a.t0, y0);
      const double dtc = a.dt ? a.dt[cell] : a.dt_scalar;
      st = g.solve_to(a.t0 + dtc);
      tc_phase = g.tc_phase;
      if (g.tc_failed) {
        tc_failed = true;
        if (tid == 0) atomicOr(err, kErrTensorCoreWait);
      }
      yf = g.y;
      nsteps = g.cnt[CNT_STEPS];
      Q = W.slot[2];
      if (tid == 0 && a.counters)
        for (int k = 0; k < NCNT; ++k) a.counters[(size_t)cell * NCNT + k] = g.cnt[k];
    } else if (tid == 0 && a.counters) {
      for (int k = 0; k < NCNT; ++k) a.counters[(size_t)cell * NCNT + k] = 0;
    }
    // solvers/laminarSMOKE/utilities.H:153-200
    const double s = bsum<BT>(tid < NC ? yf : 0., W.red);
    if (tid < NC) a.Y[(size_t)tid * a.ld + cell] = yf / s;
    if (tid == NC && o.energy) a.T[cell] = yf;
    if (tid == 0) {
      if (a.status) a.status[cell] = st;
      if (a.nsteps) a.nsteps[cell] = (int)nsteps;
      if (a.Q) a.Q[cell] = Q;
    }
  }
  if constexpr (TC) {
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid < 32) tc::tmem_dealloc(tmem, TCL ? (uint32_t)BT : (uint32_t)tc::kCols);
  }
}

// ---------------------------------------------------------------------------
// DRG-reduced step for mechanisms above 31 species (chemistry_DRG.H:86-200 with
// DRG.hpp), one block per cell, FP64 factors: the block form of drg_warp_kernel.
// Per cell above min_T: the analysis at the cell's (unclipped) state, the
// reduced system (important species and T) by a fresh solver, the kept species
// at their start values, the mass fractions normalised after the step.
// Shared memory: the block form's, then DX [BT] doubles, warp counts, the
// search queue [2 BT], the reached flags [BT] and the dropped mask [NR].
// ---------------------------------------------------------------------------
template <int BT>
__host__ __device__ inline size_t drg_block_smem(const MechLayout& L) {
  return ((block_shared_bytes<BT>(L) + 15) & ~(size_t)15) + sizeof(double) * BT + sizeof(int) * (BT / 32 + 4) +
         sizeof(int) * 3 * BT + (size_t)L.nr + 16;
}

template <int BT>
__global__ void __launch_bounds__(BT, BT == 128 ? 4 : (BT == 256 ? 2 : 1))
    drg_block_kernel(MechLayout L, const unsigned char* __restrict__ mech_gmem, StepOptions o, StepArgs a, DrgArgs d,
                     double* __restrict__ ws_all) {
  extern __shared__ __align__(16) unsigned char bsm[];
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int NC = L.nc, NR = L.nr;
  double* ws = ws_all + (size_t)blockIdx.x * block_ws_doubles(L);
  double* Jp = ws;
  double* Gp = ws + (size_t)(NC + 1) * (NC + 1);
  double* karr = ws + 2 * (size_t)(NC + 1) * (NC + 1);
  BlockShared W;
  {
    double* p = (double*)bsm;
    W.Z = p; p += 8 * BT;
    W.V = p; p += 8 * BT;
    W.C = p; p += NC;
    W.H = p; p += NC;
    W.S = p; p += NC;
    W.NET = p; p += L.nr;
    W.X = p; p += BT;
    W.red = p; p += BT / 32 + 1;
    W.slot = p; p += 4;
    W.PIV = (int*)p;
    W.ival = W.PIV + BT;
    W.PERM = W.ival + BT / 32 + 1;
  }
  unsigned char* ex = bsm + ((block_shared_bytes<BT>(L) + 15) & ~(size_t)15);
  W.DX = (double*)ex;
  int* WC = (int*)(W.DX + BT);          // per-warp counts
  int* QU = WC + (BT / 32 + 4);         // the search queue (at most nkey + NC <= 2 NC entries)
  int* IMPF = QU + 2 * BT;              // reached flags, then the reduced index -> species table
  W.DROP = (unsigned char*)(IMPF + BT);
  const MechView M{(const double*)mech_gmem, (const int*)(mech_gmem + (size_t)L.n_double * sizeof(double))};
  for (long cell = blockIdx.x; cell < a.ncells; cell += gridDim.x) {
    __syncthreads();
    const double Tc = a.T[cell];
    const double om = tid < NC ? a.Y[(size_t)tid * a.ld + cell] : 0.;
    int st = 0, nsp = 0, nrx = 0;
    if (Tc > d.min_T) {   // the same in every thread
      // ---- analysis (DRG.hpp:150-273) ----
      if (tid == 0) { W.slot[1] = 0.; W.slot[2] = 0.; }
      __syncthreads();
      rhs_block<BT>(L, M, W, karr, karr + L.nr, karr + 2 * L.nr, karr + 2 * L.nr + (L.n_fo > 0 ? L.n_fo : 1),
                    tid < NC ? om : Tc, Tc, a.p, o.energy, 0.);   // W.NET: net rates of progress
      __syncthreads();
      const double eps = d.eps[cell];
      double den = 0.;
      if (tid < NC)
        for (int k = 0; k < NR; ++k) {
          const double nki = drg_net_nu(M, L, k, tid);
          if (nki != 0.) den += fabs(nki * W.NET[k]);
        }
      W.DX[tid] = den;
      IMPF[tid] = 0;
      __syncthreads();
      if (tid == 0)
        for (int t = 0; t < d.nkey; ++t) {
          QU[t] = d.key[t];
          IMPF[d.key[t]] = 1;
        }
      __syncthreads();
      int qlen = d.nkey;
      for (int head = 0; head < qlen; ++head) {
        const int q = QU[head];
        const double denq = W.DX[q];
        double num = 0.;
        if (tid < NC)
          for (int k = 0; k < NR; ++k) {
            const double nq = drg_net_nu(M, L, k, q);
            if (nq == 0.) continue;
            if (drg_net_nu(M, L, k, tid) != 0.) num += fabs(nq * W.NET[k]);
          }
        const bool add = tid < NC && IMPF[tid] == 0 && num / (1.e-64 + denq) > eps;
        const unsigned m = __ballot_sync(kFull, add);
        if (lane == 0) WC[warp] = __popc(m);
        __syncthreads();   // every thread has read IMPF and QU for this head
        int before = 0, total = 0;
        for (int w = 0; w < BT / 32; ++w) {
          if (w < warp) before += WC[w];
          total += WC[w];
        }
        if (add) {   // appended in ascending species order
          QU[qlen + before + __popc(m & ((1u << lane) - 1u))] = tid;
          IMPF[tid] = 1;
        }
        qlen += total;
        __syncthreads();
      }
      // a reaction is dropped when one of its species (non-zero net coefficient) was not reached
      int nd = 0;
      {
        const int* pp = M.I(L.prod_ptr);
        const int* psp = M.I(L.prod_sp);
        const int* rpp = M.I(L.reac_ptr);
        const int* rsp = M.I(L.reac_sp);
        for (int k = tid; k < NR; k += BT) {
          bool keep = true;
          for (int q = pp[k]; q < pp[k + 1]; ++q) {
            const int sp = psp[q];
            if (IMPF[sp] == 0 && drg_net_nu(M, L, k, sp) != 0.) keep = false;
          }
          for (int q = rpp[k]; q < rpp[k + 1]; ++q) {
            const int sp = rsp[q];
            if (IMPF[sp] == 0 && drg_net_nu(M, L, k, sp) != 0.) keep = false;
          }
          W.DROP[k] = keep ? 0 : 1;
          nd += keep ? 0 : 1;
        }
      }
      const double ndrop = bsum<BT>((double)nd, W.red);
      // ---- the reduced system: thread l < ni owns the l-th important species, thread ni owns T ----
      const bool imp = tid < NC && IMPF[tid] != 0;
      const unsigned mi = __ballot_sync(kFull, imp);
      __syncthreads();
      if (lane == 0) WC[warp] = __popc(mi);
      __syncthreads();
      int before = 0, ni = 0;
      for (int w = 0; w < BT / 32; ++w) {
        if (w < warp) before += WC[w];
        ni += WC[w];
      }
      const int pos = imp ? before + __popc(mi & ((1u << lane) - 1u)) : -1;
      W.DX[tid] = om;   // full layout: the start mass fractions
      __syncthreads();
      if (imp) QU[pos] = tid;   // reduced index -> species
      __syncthreads();
      const int sp = tid < ni ? QU[tid] : NC;
      const double y0 = tid < ni ? W.DX[sp] : (tid == ni ? Tc : 0.);
      __syncthreads();
      GearBlock<BT, false, true> g;
      g.L = &L;
      g.M = M;
      g.W = W;
      g.J = Jp;
      g.jld = NC + 1;
      g.G = Gp;
      g.karr = karr;
      g.ukeq = g.karr + L.nr;
      g.kinf = g.ukeq + L.nr;
      g.logf = g.kinf + (L.n_fo > 0 ? L.n_fo : 1);
      g.P0 = a.p;
      g.rho0 = 0.;
      g.energy = o.energy;
      g.tid = tid;
      g.ne = ni + 1;
      g.active = tid < ni + 1;
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
        g.minv = tid < ni ? 0. : 200.;
        g.maxv = tid < ni ? 1. : 6000.;
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
      if (tid == 0) { W.slot[1] = 0.; }
      __syncthreads();
      g.set_initial_conditions(a.t0, y0);
      const double dtc = a.dt ? a.dt[cell] : a.dt_scalar;
      st = g.solve_to(a.t0 + dtc);
      // ---- scatter: the kept species' start values, the integrated ones, T; normalised ----
      __syncthreads();
      W.DX[tid] = g.y;   // reduced layout
      __syncthreads();
      const double Tf = W.DX[ni];
      const double yf = pos >= 0 ? W.DX[pos] : om;
      const double sum = bsum<BT>(tid < NC ? yf : 0., W.red);
      if (tid < NC) a.Y[(size_t)tid * a.ld + cell] = yf / sum;
      if (tid == 0) {
        if (o.energy) a.T[cell] = Tf;
        if (a.Q) a.Q[cell] = W.slot[2];
        if (a.counters)
          for (int k = 0; k < NCNT; ++k) a.counters[(size_t)cell * NCNT + k] = g.cnt[k];
        if (a.nsteps) a.nsteps[cell] = (int)g.cnt[CNT_STEPS];
      }
      nsp = ni;
      nrx = NR - (int)ndrop;
    } else if (tid == 0) {
      if (a.counters)
        for (int k = 0; k < NCNT; ++k) a.counters[(size_t)cell * NCNT + k] = 0;
      if (a.nsteps) a.nsteps[cell] = 0;
    }
    if (tid == 0) {
      if (a.status) a.status[cell] = st;
      if (d.n_species) d.n_species[cell] = nsp;
      if (d.n_reactions) d.n_reactions[cell] = nrx;
    }
  }
}

// ---------------------------------------------------------------------------
// Stand-alone tensor-core inverse (lsg_build_and_invert_g_device): persistent
// blocks of 128 threads, one matrix at a time; G^-1 written column-major FP32.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 2) tc_inverse_kernel(int nmat, int n, const double* __restrict__ J,
                                                            const double* __restrict__ hr0, float* __restrict__ out,
                                                            int* err) {
  extern __shared__ __align__(16) unsigned char tsm[];
  const int tid = threadIdx.x;
  const uint32_t s0 = tc::smem_addr(tsm);
  unsigned char* q = tsm + (((s0 + 1023u) & ~1023u) - s0);
  tc::Smem TS{};
  TS.op = (float*)q; q += 4 * tc::kOperandFloats * sizeof(float);
  TS.mbar = (unsigned long long*)q; q += 16;
  TS.tmem_slot = (uint32_t*)q; q += 16;
  TS.red = (float*)q; q += 8 * sizeof(float);
  TS.redi = (int*)q; q += 8 * sizeof(int);
  TS.prow = (float*)q; q += 4 * tc::kPanel * sizeof(float);
  TS.pivot_of_row = (int*)q;
  if (tid < 32) tc::tmem_alloc(TS.tmem_slot, tc::kCols);
  if (tid == 0) tc::mbar_init(TS.mbar, 1);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *TS.tmem_slot;
  uint32_t phase = 0;
  for (int m = blockIdx.x; m < nmat; m += gridDim.x) {
    if (!tc::gj_inverse(J + (size_t)m * n * n, n, hr0[m], TS, tmem, &phase)) {
      if (tid == 0) atomicOr(err, kErrTensorCoreWait);
      break;
    }
    float* o = out + (size_t)m * n * n;
    for (int e = tid; e < n * n; e += 128) {
      const int j = e / n, c = e - j * n;
      o[e] = TS.op[j * tc::kRows + c];
    }
    __syncthreads();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (tid < 32) tc::tmem_dealloc(tmem, tc::kCols);
}

// Stand-alone multi-tile inverse (128 < n <= 512): blocks of BT = 128 MT threads, each with an FP32 work
// matrix of BT x BT in ws; G^-1[a][b] = R[c(b) * BT + p_a] (gj_inverse_large) written column-major FP32.
template <int BT>
__host__ __device__ inline size_t tcl_inverse_smem() {
  return 1024 + sizeof(float) * ((2 * (BT / 128) + 2) * (size_t)tc::kOperandFloats + 64 + 4 * tc::kPanel) +
         sizeof(int) * 2 * BT + 64;
}

template <int MT>
__global__ void __launch_bounds__(MT * 128, 1) tc_inverse_large_kernel(int nmat, int n, const double* __restrict__ J,
                                                                       const double* __restrict__ hr0,
                                                                       float* __restrict__ out, float* __restrict__ ws,
                                                                       int* err) {
  constexpr int BT = MT * 128;
  extern __shared__ __align__(16) unsigned char tsm[];
  __shared__ uint32_t tslot;
  __shared__ __align__(8) unsigned long long mbar;
  const int tid = threadIdx.x;
  const uint32_t s0 = tc::smem_addr(tsm);
  unsigned char* q = tsm + (((s0 + 1023u) & ~1023u) - s0);
  tc::SmemL TL{};
  TL.A = (float*)q;
  TL.B = TL.A + 2 * MT * tc::kOperandFloats;
  float* f = TL.B + 2 * tc::kOperandFloats;
  TL.red = f; f += 32;
  TL.redi = (int*)f; f += 32;
  TL.prow = f; f += 4 * tc::kPanel;
  TL.piv = (int*)f;
  TL.colof = TL.piv + BT;
  TL.mbar = &mbar;
  if (tid < 32) tc::tmem_alloc(&tslot, BT);
  if (tid == 0) tc::mbar_init(&mbar, 1);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tslot;
  uint32_t phase = 0;
  float* R = ws + (size_t)blockIdx.x * BT * BT;
  for (int m = blockIdx.x; m < nmat; m += gridDim.x) {
    if (!tc::gj_inverse_large<MT>(J + (size_t)m * n * n, n, n, hr0[m], R, TL, tmem, &phase)) {
      if (tid == 0) atomicOr(err, kErrTensorCoreWait);
      break;
    }
    float* o = out + (size_t)m * n * n;
    for (int e = tid; e < n * n; e += BT) {
      const int b = e / n, a = e - b * n;   // element (a, b) of G^-1
      o[e] = R[(size_t)TL.colof[b] * BT + TL.piv[a]];
    }
    __syncthreads();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (tid < 32) tc::tmem_dealloc(tmem, BT);
}

// ---------------------------------------------------------------------------
// Stand-alone RHS for large mechanisms: one block per state (the same
// arithmetic as inside the block step).  y/dy species-major [(NC+1) * ld].
// ---------------------------------------------------------------------------
template <int BT>
__global__ void __launch_bounds__(BT) rhs_block_kernel(MechLayout L, const unsigned char* __restrict__ mech_gmem,
                                                       long ncells, const double* __restrict__ y,
                                                       double* __restrict__ dy, long ld, double p, int energy,
                                                       double* qr, double* __restrict__ ws_all) {
  extern __shared__ __align__(16) unsigned char bsm[];
  const int tid = threadIdx.x;
  const int NC = L.nc;
  double* ws = ws_all + (size_t)blockIdx.x * block_ws_doubles(L);
  const size_t n = NC + 1;
  double* karr = ws + 2 * n * n;
  double* ukeq = karr + L.nr;
  double* kinf = ukeq + L.nr;
  double* logf = kinf + (L.n_fo > 0 ? L.n_fo : 1);
  BlockShared W;
  {
    double* q = (double*)bsm;
    W.Z = q; q += 8 * BT;
    W.V = q; q += 8 * BT;
    W.C = q; q += NC;
    W.H = q; q += NC;
    W.S = q; q += NC;
    W.NET = q; q += L.nr;
    W.X = q; q += BT;
    W.red = q; q += BT / 32 + 1;
    W.slot = q; q += 4;
    W.PIV = (int*)q;
    W.ival = W.PIV + BT;
    W.PERM = W.ival + BT / 32 + 1;
  }
  const MechView M{(const double*)mech_gmem, (const int*)(mech_gmem + (size_t)L.n_double * sizeof(double))};
  for (long cell = blockIdx.x; cell < ncells; cell += gridDim.x) {
    __syncthreads();
    if (tid == 0) { W.slot[1] = 0.; W.slot[2] = 0.; }
    const double yl = tid <= NC ? y[(size_t)tid * ld + cell] : 0.;
    const double T = bcast(yl, NC, W.slot);
    const double d = rhs_block<BT>(L, M, W, karr, ukeq, kinf, logf, yl, T, p, energy, 0.);
    if (tid <= NC) dy[(size_t)tid * ld + cell] = d;
    if (tid == 0 && qr) qr[cell] = W.slot[2];
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

// Shared memory of the mixed-precision (tensor-core) block kernel: the FP64 form's, then the inverse's
// operands (64 KB, 1024-byte aligned) and small arrays; at least 80 KB so that at most two blocks share
// an SM (each holds 256 of the SM's 512 TMEM columns).
size_t tc_block_smem(const MechLayout& L) {
  const size_t base = block_shared_bytes<128>(L) + 1024;   // + the alignment of the operands
  const size_t s = base + 4 * tc::kOperandFloats * sizeof(float) + 32 + 16 * sizeof(float) +
                   4 * tc::kPanel * sizeof(float) + tc::kRows * sizeof(int);
  return s < 80 * 1024 ? 80 * 1024 : s;
}

template <int BT, bool TC>
size_t block_smem(const MechLayout& L) {
  if (!TC) return block_shared_bytes<BT>(L);
  return BT == 128 ? tc_block_smem(L) : tcl_smem_bytes<BT>(L);
}

template <int BT, bool TC>
cudaError_t block_setup(const MechLayout& L, size_t* smem, int* bps) {
  *smem = block_smem<BT, TC>(L);
  if (*smem > 227 * 1024) return cudaErrorInvalidConfiguration;
  cudaError_t e = cudaFuncSetAttribute(block_kernel<BT, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, block_kernel<BT, TC>, BT, *smem);
  // TMEM: 256 columns a block up to 128 components, BT columns above (512 on the SM)
  const int tmem_cap = BT == 128 ? 2 : 512 / BT;
  if (TC && *bps > tmem_cap) *bps = tmem_cap;
  return e;
}

int block_threads(const MechLayout& L) { return block_bt(L.nc + 1); }

}  // namespace

cudaError_t upload_gear_block(const GearConsts& gc) { return cudaMemcpyToSymbol(c_gear_k, &gc, sizeof(GearConsts)); }

size_t block_ws_bytes(const MechLayout& L) { return block_ws_doubles(L) * sizeof(double); }

bool block_tc_eligible(const MechLayout& L) {
  const int n = L.nc + 1;
  if (n < 32 || n > kBlkMaxN) return false;
  const int bt = block_bt(n);
  const size_t smem = bt == 128 ? tc_block_smem(L) : (bt == 256 ? tcl_smem_bytes<256>(L) : tcl_smem_bytes<512>(L));
  return smem <= 227 * 1024;
}

cudaError_t block_plan(const MechLayout& L, int sm_count, bool tc, long* nblocks) {
  if (L.nc + 1 > kBlkMaxN) return cudaErrorInvalidValue;
  if (tc && !block_tc_eligible(L)) return cudaErrorInvalidValue;
  size_t smem = 0;
  int bps = 0;
  const int bt = block_threads(L);
  cudaError_t e = tc ? (bt == 128 ? block_setup<128, true>(L, &smem, &bps)
                                   : (bt == 256 ? block_setup<256, true>(L, &smem, &bps)
                                                : block_setup<512, true>(L, &smem, &bps)))
                     : (bt == 128 ? block_setup<128, false>(L, &smem, &bps)
                                  : (bt == 256 ? block_setup<256, false>(L, &smem, &bps)
                                               : block_setup<512, false>(L, &smem, &bps)));
  if (e != cudaSuccess) return e;
  if (bps <= 0 || smem > 227 * 1024) return cudaErrorInvalidConfiguration;
  *nblocks = (long)sm_count * bps;
  return cudaSuccess;
}

cudaError_t launch_block(const MechLayout& L, const unsigned char* mech_gmem, const StepOptions& o,
                         const StepArgs& a, double* ws, long nblocks, int* queue, bool tc, int* err,
                         cudaStream_t stream) {
  if (a.ncells <= 0) return cudaSuccess;
  long g = nblocks < a.ncells ? nblocks : a.ncells;
  cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(int), stream);
  if (e != cudaSuccess) return e;
  const int bt = block_threads(L);
  if (tc) {
    if (!block_tc_eligible(L)) return cudaErrorInvalidValue;
    if (bt == 128)
      block_kernel<128, true><<<(unsigned)g, 128, block_smem<128, true>(L), stream>>>(L, mech_gmem, o, a, ws, queue, err);
    else if (bt == 256)
      block_kernel<256, true><<<(unsigned)g, 256, block_smem<256, true>(L), stream>>>(L, mech_gmem, o, a, ws, queue, err);
    else
      block_kernel<512, true><<<(unsigned)g, 512, block_smem<512, true>(L), stream>>>(L, mech_gmem, o, a, ws, queue, err);
  } else if (bt == 128) {
    block_kernel<128, false><<<(unsigned)g, 128, block_shared_bytes<128>(L), stream>>>(L, mech_gmem, o, a, ws, queue, err);
  } else if (bt == 256) {
    block_kernel<256, false><<<(unsigned)g, 256, block_shared_bytes<256>(L), stream>>>(L, mech_gmem, o, a, ws, queue, err);
  } else {
    block_kernel<512, false><<<(unsigned)g, 512, block_shared_bytes<512>(L), stream>>>(L, mech_gmem, o, a, ws, queue, err);
  }
  return cudaGetLastError();
}

size_t tc_inverse_smem() {
  return 1024 + 4 * tc::kOperandFloats * sizeof(float) + 32 + 16 * sizeof(float) + 4 * tc::kPanel * sizeof(float) +
         tc::kRows * sizeof(int);
}

size_t tc_inverse_ws_bytes(int n, int sm_count) {
  if (n <= tc::kRows) return 0;
  const size_t np = (size_t)block_bt(n);
  return np * np * sizeof(float) * (size_t)sm_count * (512 / np);
}

template <int MT>
cudaError_t launch_tc_inverse_large(int nmat, int n, const double* J, const double* hr0, float* out, float* ws,
                                    int sm_count, int* err, cudaStream_t stream) {
  constexpr int BT = MT * 128;
  const size_t smem = tcl_inverse_smem<BT>();
  cudaError_t e =
      cudaFuncSetAttribute(tc_inverse_large_kernel<MT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const long cap = (long)sm_count * (512 / BT);
  const long g = cap < nmat ? cap : nmat;
  tc_inverse_large_kernel<MT><<<(unsigned)g, BT, smem, stream>>>(nmat, n, J, hr0, out, ws, err);
  return cudaGetLastError();
}

cudaError_t launch_tc_inverse(int nmat, int n, const double* J, const double* hr0, float* out, float* ws,
                              int sm_count, int* err, cudaStream_t stream) {
  if (n < 1 || n > kBlkMaxN || nmat < 0) return cudaErrorInvalidValue;
  if (nmat == 0) return cudaSuccess;
  if (n > tc::kRows) {
    if (!ws) return cudaErrorInvalidValue;
    return n <= 256 ? launch_tc_inverse_large<2>(nmat, n, J, hr0, out, ws, sm_count, err, stream)
                    : launch_tc_inverse_large<4>(nmat, n, J, hr0, out, ws, sm_count, err, stream);
  }
  size_t smem = tc_inverse_smem();
  if (smem < 80 * 1024) smem = 80 * 1024;   // at most two blocks per SM: 256 TMEM columns each
  cudaError_t e = cudaFuncSetAttribute(tc_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const long g = (long)sm_count * 2 < nmat ? (long)sm_count * 2 : nmat;
  tc_inverse_kernel<<<(unsigned)g, 128, smem, stream>>>(nmat, n, J, hr0, out, err);
  return cudaGetLastError();
}

cudaError_t launch_rhs_block(const MechLayout& L, const unsigned char* mech_gmem, long ncells, const double* y,
                             double* dy, long ld, double p, int energy, double* qr, double* ws, long nblocks,
                             cudaStream_t stream) {
  if (ncells <= 0) return cudaSuccess;
  const long g = nblocks < ncells ? nblocks : ncells;
  const int bt = block_threads(L);
  cudaError_t e;
  if (bt == 128) {
    e = cudaFuncSetAttribute(rhs_block_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)block_shared_bytes<128>(L));
    if (e != cudaSuccess) return e;
    rhs_block_kernel<128><<<(unsigned)g, 128, block_shared_bytes<128>(L), stream>>>(L, mech_gmem, ncells, y, dy, ld,
                                                                                     p, energy, qr, ws);
  } else if (bt == 256) {
    e = cudaFuncSetAttribute(rhs_block_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)block_shared_bytes<256>(L));
    if (e != cudaSuccess) return e;
    rhs_block_kernel<256><<<(unsigned)g, 256, block_shared_bytes<256>(L), stream>>>(L, mech_gmem, ncells, y, dy, ld,
                                                                                     p, energy, qr, ws);
  } else {
    e = cudaFuncSetAttribute(rhs_block_kernel<512>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)block_shared_bytes<512>(L));
    if (e != cudaSuccess) return e;
    rhs_block_kernel<512><<<(unsigned)g, 512, block_shared_bytes<512>(L), stream>>>(L, mech_gmem, ncells, y, dy, ld,
                                                                                     p, energy, qr, ws);
  }
  return cudaGetLastError();
}

template <int BT>
cudaError_t drg_block_launch(const MechLayout& L, const unsigned char* mech_gmem, const StepOptions& o,
                             const StepArgs& a, const DrgArgs& d, double* ws, long nblocks, cudaStream_t stream) {
  const size_t smem = drg_block_smem<BT>(L);
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(drg_block_kernel<BT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const long g = nblocks < a.ncells ? nblocks : a.ncells;
  drg_block_kernel<BT><<<(unsigned)g, BT, smem, stream>>>(L, mech_gmem, o, a, d, ws);
  return cudaGetLastError();
}

cudaError_t launch_drg_block(const MechLayout& L, const unsigned char* mech_gmem, const StepOptions& o,
                             const StepArgs& a, const DrgArgs& d, double* ws, long nblocks, cudaStream_t stream) {
  if (a.ncells <= 0) return cudaSuccess;
  if (L.nc + 1 > kBlkMaxN || nblocks <= 0) return cudaErrorInvalidValue;
  const int bt = block_threads(L);
  if (bt == 128) return drg_block_launch<128>(L, mech_gmem, o, a, d, ws, nblocks, stream);
  if (bt == 256) return drg_block_launch<256>(L, mech_gmem, o, a, d, ws, nblocks, stream);
  return drg_block_launch<512>(L, mech_gmem, o, a, d, ws, nblocks, stream);
}

}  // namespace lsg
