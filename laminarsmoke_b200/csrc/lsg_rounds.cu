// Batched reaction step, round scheme: every cell of the batch is one
// thread-sized state machine with its whole state in HBM (structure of arrays,
// [field][cell], so a warp's accesses are coalesced); the step advances in
// rounds, each a fixed sequence of throughput kernels over the list of cells
// still integrating:
//
//   rhs       one thread per cell evaluates the RHS the cell asked for
//             (f(y0), the predictor, a finite-difference Jacobian column, a
//             Newton iterate, a stabilisation call or the final call at tOut);
//             mechanism tables staged into shared memory by a bulk copy;
//   advance   one thread per cell consumes the result and runs the cell's
//             Gear/BDF solver until its next RHS request, a factorisation
//             request, or the end of its integration;
//   factor    one warp per requested factorisation: G = I - h r0 J, partial
//             pivoting, factors in FP32 (mixed precision) or FP64;
//   advance   cells that were just factorised continue to their next RHS
//             request;
//   compact   the cells that are still integrating form the next round's
//             list (order-preserving inside each warp).
//
// Each kernel keeps many warps in flight (little per-cell on-chip state), so the
// latency of the solver's scattered control flow is hidden by occupancy instead
// of being paid once per thread.  The method is the one of the plain step --
// MultiValueSolver.hpp:423-1328, MethodGear.hpp:195-516, KernelDense.hpp:111-193
// (under solvers/openSMOKEpp4laminarSMOKE/math/native-ode-solvers) -- with the
// RHS of BatchReactorHomogeneousConstantPressure.H:175-223.  With FP32 factors
// every linear solve is refined against its FP64 residual (the matrix rebuilt in
// FP64 from the stored Jacobian) until it equals the FP64 solve to rounding.
#include "lsg_common.cuh"
#include "lsg_kernels.h"

namespace lsg {

static __constant__ GearConsts c_gear_r;

namespace {

constexpr int kRT = 128;       // threads per block of the RHS kernel (one cell each)
constexpr int kAT = 128;       // threads per block of the advance kernel
constexpr int kFW = 4;         // warps per block of the factor kernel
constexpr int kCT = 256;       // threads per block of the compaction kernel
constexpr int kRefineR = 2;    // refinement sweeps of a solve with FP32 factors

enum Phase : int {
  PH_DONE = 0,
  PH_INIT,       // f(y0)
  PH_PRED,       // f(vb), first Newton evaluation
  PH_JAC,        // f(vb + hJ e_j), FD column jcol
  PH_NEWTON,     // f(va), Newton iterate
  PH_STAB_CONV,  // f(z0) during convergence-failure recovery
  PH_STAB_ERR,   // f(z0) after an error-test failure
  PH_FINAL,      // f(y(tOut)) -> QR
  PH_FACT,       // waiting for the factorisation of G
  PH_FACTORED,   // factorised, continue after FindCorrection's factorisation
};

__device__ __forceinline__ bool rhs_phase(int ph) { return ph >= PH_INIT && ph <= PH_FINAL; }

// scalar state of a cell: doubles [D_*][ns], ints [I_*][ns]
enum : int {
  D_T = 0, D_T0, D_TOUT, D_TMESH, D_TSTAB, D_H, D_HNEXT, D_HNORD, D_HSCALE, D_HSCALEMAX,
  D_A24, D_A25, D_QR, D_OLDCC, D_HF, D_HJ, D_PENDHS, D_HR0, ND_
};
enum : int {
  I_PHASE = 0, I_STATUS, I_P, I_ITORDER, I_ORDNEXT, I_MAXITJ, I_HSTAT, I_OSTAT, I_FACTORIZED, I_JACCHANGE,
  I_CONVOK, I_NSTEPS, I_ITCONV, I_ITCONVRATE, I_ITCONVFAIL, I_ITERRFAIL, I_NCFOM, I_STEPLASTJ, I_ITCONST,
  I_ITMINORD, I_FIXEDMIN, I_NEWTONK, I_JCOL, I_MAXORD, I_CNT0, NI_ = I_CNT0 + NCNT
};

__device__ __forceinline__ double contrib_r(double nu, double v) {
  if (nu == 1.) return v;
  if (nu == 2.) return v + v;
  if (nu == 3.) return v + v + v;
  if (nu == 0.5) return 0.5 * v;
  return nu * v;
}

__device__ __forceinline__ double conc_factor_r(double nu, double c1) {
  if (nu == 1.) return c1;
  if (nu == 2.) return c1 * c1;
  if (nu == 3.) return c1 * c1 * c1;
  if (nu == 0.5) return sqrt(c1);
  return pow(c1, nu);
}

__device__ __forceinline__ double lo_b(int k, int NC, double yminT) { return k < NC ? 0. : yminT; }
__device__ __forceinline__ double hi_b(int k, int NC, double ymaxT) { return k < NC ? 1. : ymaxT; }

// ---------------------------------------------------------------------------
// Thread-serial RHS of the constant-pressure reactor
// (BatchReactorHomogeneousConstantPressure.H:175-223).  y: this cell's input
// vector (stride ns) with component pj replaced by pval when pj >= 0; f: output.
// C,H,S,R scratch in shared memory, [species][thread].  Returns QR.
// ---------------------------------------------------------------------------
__device__ __noinline__ double rhs_cell(const MechLayout* __restrict__ Lp, const double* __restrict__ Md,
                                        const int* __restrict__ Mi, double* __restrict__ scratch,
                                        const double* __restrict__ y, long ns, int pj, double pval,
                                        double* __restrict__ f, double P0, int energy) {
  const MechLayout& L = *Lp;
  const MechView M{Md, Mi};
  const int NC = L.nc, NR = L.nr;
  const int tid = threadIdx.x;
  double* C = scratch;
  double* H = scratch + NC * kRT;
  double* Sx = scratch + 2 * NC * kRT;
  double* R = scratch + 3 * NC * kRT;
#define SC_(arr, i) arr[(i) * kRT + tid]
  const double* MW = M.D(L.mw);
  const double T = (pj == NC) ? pval : y[(long)NC * ns];
  double u = 0.;
#pragma unroll 4
  for (int i = 0; i < NC; ++i) {
    const double yi = (i == pj) ? pval : y[(long)i * ns];
    SC_(C, i) = yi;
    u += yi / MW[i];
  }
  const double MWmix = 1. / u;
  const double cTot = P0 / kRgas / T;
  const double rho = cTot * MWmix;
  const double* TM = M.D(L.t_mid);
  const double T2 = T * T, T3 = T2 * T, T4 = T3 * T, uT = 1. / T;
  const double logT = log(T);
  const double lP = log(101325. / kRgas / T);
  double cTotSum = 0.;
  for (int i = 0; i < NC; ++i) {
    double x = MWmix * SC_(C, i);
    x = x / MW[i];
    const double c = cTot * x;
    SC_(C, i) = c;
    cTotSum += c;
    const bool hi = T > TM[i];
    const double* A = hi ? M.D(L.dh_ht) + 6 * i : M.D(L.dh_lt) + 6 * i;
    SC_(H, i) = A[0] + T * A[1] + T2 * A[2] + T3 * A[3] + T4 * A[4] + uT * A[5];
    const double* B = hi ? M.D(L.ds_ht) + 6 * i : M.D(L.ds_lt) + 6 * i;
    SC_(Sx, i) = B[0] * logT + T * B[1] + T2 * B[2] + T3 * B[3] + T4 * B[4] + B[5];
    SC_(R, i) = 0.;
  }
  const double* lnA = M.D(L.lnA);
  const double* beta = M.D(L.beta);
  const double* eor = M.D(L.eor);
  const double* dnu = M.D(L.dnu);
  const int* sgn = M.I(L.a_sign);
  const int* rk = M.I(L.rev_kind);
  const int* rs = M.I(L.rev_slot);
  const int* tbs = M.I(L.tb_slot);
  const int* fos = M.I(L.fo_slot);
  const int* rp = M.I(L.reac_ptr);
  const int* rsp = M.I(L.reac_sp);
  const double* rnu = M.D(L.reac_nu);
  const int* pp = M.I(L.prod_ptr);
  const int* psp = M.I(L.prod_sp);
  const double* pnu = M.D(L.prod_nu);
  for (int j = 0; j < NR; ++j) {
    double kArr = exp(lnA[j] + beta[j] * logT - eor[j] * uT);
    if (sgn[j] < 0) kArr *= -1.;
    double kMod = kArr;
    const int tb = tbs[j];
    if (tb >= 0) {
      double Mc = cTotSum;
      const int* tp = M.I(L.tb_ptr);
      const int* ts = M.I(L.tb_sp);
      const double* te = M.D(L.tb_eff);
      for (int q = tp[tb]; q < tp[tb + 1]; ++q) Mc += SC_(C, ts[q]) * te[q];
      kMod *= Mc;
    }
    const int fo = fos[j];
    if (fo >= 0) {
      // KineticsMap_CHEMKIN::KineticConstants fall-off part (:1257-1290) and FallOffReactions (:1496-1550)
      const double kInf = exp(M.D(L.fo_lnA)[fo] + M.D(L.fo_beta)[fo] * logT - M.D(L.fo_eor)[fo] * uT);
      const double a = M.D(L.fo_a)[fo], b = M.D(L.fo_b)[fo], c = M.D(L.fo_c)[fo], d = M.D(L.fo_d)[fo];
      const int ty = M.I(L.fo_type)[fo];
      double Mc;
      const int single = M.I(L.fo_single)[fo];
      if (single < 0) {
        Mc = cTotSum;
        const int* fp = M.I(L.fo_ptr);
        const int* fs = M.I(L.fo_sp);
        const double* fe = M.D(L.fo_eff);
        for (int q = fp[fo]; q < fp[fo + 1]; ++q) Mc += SC_(C, fs[q]) * fe[q];
      } else {
        Mc = SC_(C, single) + 1.e-16;
      }
      const double Pr = kArr * Mc / kInf;
      double wF = 1.;
      if (ty == 1) {
        double v = (1. - a) * exp(-T / b) + a * exp(-T / c);
        if (d != 0.) v += exp(-d / T);
        const double lF = (v < 1.e-300) ? -300. : log10(v);
        double qq;
        if (Pr > 1.e-32) {
          const double nTroe = 0.75 - 1.27 * lF;
          const double cTroe = -0.4 - 0.67 * lF;
          const double sTroe = log10(Pr) + cTroe;
          qq = sTroe / (nTroe - 0.14 * sTroe);
        } else {
          qq = 1. / 0.14;
        }
        wF = exp10(lF / (1. + qq * qq));
      } else if (ty == 2) {
        const double lF = a * exp(-b / T) + exp(-T / c);
        const double l10 = log10(Pr);
        const double xSRI = 1. / (1. + l10 * l10);
        wF = pow(lF, xSRI) * d;
        const double e = M.D(L.fo_e)[fo];
        if (e != 0.) wF *= pow(T, e);
      }
      kMod *= kInf * (Pr / (1. + Pr)) * wF / kArr;
    }
    double fwd = 1.;
    for (int q = rp[j]; q < rp[j + 1]; ++q) fwd *= conc_factor_r(rnu[q], SC_(C, rsp[q]));
    double net = fwd;
    const int kind = rk[j];
    if (kind != 0) {
      double rv = 1.;
      for (int q = pp[j]; q < pp[j + 1]; ++q) rv *= conc_factor_r(pnu[q], SC_(C, psp[q]));
      if (kind == 1) {
        // 1/Keq from reaction enthalpy and entropy (StoichiometricMap.hpp:916-1001, KineticsMap_CHEMKIN.hpp:1217-1222)
        double dh = 0., ds = 0.;
        int qa = rp[j], qb = pp[j];
        const int ae = rp[j + 1], be = pp[j + 1];
        while (qa < ae || qb < be) {
          const int sa = qa < ae ? rsp[qa] : (1 << 30);
          const int sb = qb < be ? psp[qb] : (1 << 30);
          if (sa <= sb) {
            dh -= contrib_r(rnu[qa], SC_(H, sa));
            ds -= contrib_r(rnu[qa], SC_(Sx, sa));
            ++qa;
          } else {
            dh += contrib_r(pnu[qb], SC_(H, sb));
            ds += contrib_r(pnu[qb], SC_(Sx, sb));
            ++qb;
          }
        }
        rv *= exp(-ds + dh - lP * dnu[j]);
      } else {
        const int s = rs[j];
        rv *= exp(M.D(L.rev_lnA)[s] + M.D(L.rev_beta)[s] * logT - M.D(L.rev_eor)[s] * uT) / kArr;
      }
      net -= rv;
    }
    net *= kMod;
    for (int q = rp[j]; q < rp[j + 1]; ++q) SC_(R, rsp[q]) -= contrib_r(rnu[q], net);
    for (int q = pp[j]; q < pp[j + 1]; ++q) SC_(R, psp[q]) += contrib_r(pnu[q], net);
  }
  double QR = 0., cpm = 0., dsum = 0.;
  for (int i = 0; i < NC; ++i) {
    const double Ri = SC_(R, i);
    f[(long)i * ns] = MW[i] * Ri / rho;
    if (energy) {
      const double* A = (T > TM[i]) ? M.D(L.cp_ht) + 5 * i : M.D(L.cp_lt) + 5 * i;
      const double cpi = A[0] + T * A[1] + T2 * A[2] + T3 * A[3] + T4 * A[4];
      cpm += cpi * (SC_(C, i) / cTot);
      dsum += Ri * SC_(H, i);
    }
  }
  double dT = 0.;
  if (energy) {
    cpm *= kRgas;
    const double CpMixMass = cpm / MWmix;
    QR = -dsum * kRgas * T;
    dT = QR / (rho * CpMixMass);
  }
  f[(long)NC * ns] = dT;
#undef SC_
  return QR;
}

// ---------------------------------------------------------------------------
// Per-cell vector helpers.  Pointers address element 0 of a cell's vector;
// element k is at [k * ns].  __restrict__ lets each loop keep all its loads in
// flight at once (the vectors never overlap).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double wrms_r(const double* __restrict__ x, const double* __restrict__ e, int n, long ns) {
  double s = 0.;
#pragma unroll 4
  for (int k = 0; k < n; ++k) {
    const double c = x[k * ns] * e[k * ns];
    s += c * c;
  }
  return sqrt(s / double(n));
}

__device__ __forceinline__ void set_eps_r(const double* __restrict__ w, double* __restrict__ e, int n, long ns,
                                        double atol, double rtol) {
#pragma unroll 4
  for (int k = 0; k < n; ++k) e[k * ns] = 1. / (atol + rtol * fabs(w[k * ns]));
}

// DriverStep rescale of z[1..p] and CheckConstraints(z0) (MultiValueSolver.hpp:780-797)
__device__ __forceinline__ void rescale_z_r(double* __restrict__ z, int n, long ns, unsigned p, double hScale, int NC,
                                          double yminT, double ymaxT) {
  double hr = 1.;
  for (unsigned i = 1; i <= p; ++i) {
    hr *= hScale;
    double* zi = z + (long)i * n * ns;
#pragma unroll 4
    for (int k = 0; k < n; ++k) zi[k * ns] *= hr;
  }
#pragma unroll 4
  for (int k = 0; k < n; ++k) {
    double z0 = z[k * ns];
    const double lo = lo_b(k, NC, yminT), hi = hi_b(k, NC, ymaxT);
    if (z0 < lo) z0 = lo;
    if (z0 > hi) z0 = hi;
    z[k * ns] = z0;
  }
}

// MultiValueStep prediction v = D z with min/max handling (MultiValueSolver.hpp:1214-1262) and
// FindCorrection's vb = CheckConstraints(v0) (MethodGear.hpp:198-202)
__device__ __forceinline__ void predict_r(const double* __restrict__ z, double* __restrict__ v,
                                        double* __restrict__ vb, const double* __restrict__ e, int n, long ns,
                                        unsigned p, int NC, double yminT, double ymaxT) {
  for (int k = 0; k < n; ++k) {
    double w[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) w[i] = (i <= (int)p) ? z[((long)i * n + k) * ns] : 0.;
#pragma unroll
    for (int i = 0; i < 7; ++i)
#pragma unroll
      for (int j = 6; j >= 0; --j)
        if (i < (int)p && j >= i && j <= (int)p - 1) w[j] += w[j + 1];
    const double lo = lo_b(k, NC, yminT), hi = hi_b(k, NC, ymaxT);
    const double ek = e[k * ns];
    const double z0 = z[k * ns];
    if (w[0] < lo && fabs(w[0] - lo) * ek < double(n)) {
      w[1] = lo - z0;
      w[0] = lo;
#pragma unroll
      for (int i = 2; i < 8; ++i) w[i] = 0.;
    }
    if (w[0] > hi && fabs(w[0] - hi) * ek < double(n)) {
      w[1] = hi - z0;
      w[0] = hi;
#pragma unroll
      for (int i = 2; i < 8; ++i) w[i] = 0.;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i)
      if (i <= (int)p) v[((long)i * n + k) * ns] = w[i];
    double b = w[0];
    if (b < lo) b = lo;
    if (b > hi) b = hi;
    vb[k * ns] = b;
  }
}


// Forward and back substitution with factors of P G = L U (row-permuted right
// hand side already in x); column-oriented as KernelDense::SolveLinearSystem.
// x: this thread's vector in shared memory, element k at x[k * kAT].
template <typename LUT>
__device__ __forceinline__ void lu_fwd_bwd(double* __restrict__ x, const LUT* __restrict__ lu, int n, long ns) {
  for (int j = 0; j < n; ++j) {
    const double xj = x[j * kAT];
#pragma unroll 4
    for (int i = j + 1; i < n; ++i) x[i * kAT] -= (double)lu[(long)(i * n + j) * ns] * xj;
  }
  for (int j = n - 1; j >= 0; --j) {
    const double xj = x[j * kAT] / (double)lu[(long)(j * n + j) * ns];
    x[j * kAT] = xj;
#pragma unroll 4
    for (int i = 0; i < j; ++i) x[i * kAT] -= (double)lu[(long)(i * n + j) * ns] * xj;
  }
}

// x <- G^-1 r for the cell's last factorisation (r in global memory, natural
// order; perm maps factor rows to rows of G).  FP32 factors: kRefineR sweeps of
// iterative refinement on the FP64 residual r - (I - hr0 J) x.  d: second
// shared-memory vector, tmp: global scratch vector.
template <typename LUT>
__device__ __forceinline__ void lin_solve_r(double* __restrict__ x, double* __restrict__ d,
                                            const double* __restrict__ r, const LUT* __restrict__ lu,
                                            const int* __restrict__ perm, const float* __restrict__ jac,
                                            double* __restrict__ tmp, double hr0, int n, long ns) {
#pragma unroll 4
  for (int k = 0; k < n; ++k) x[k * kAT] = r[(long)perm[k * ns] * ns];
  lu_fwd_bwd<LUT>(x, lu, n, ns);
  if (sizeof(LUT) == sizeof(float)) {
    for (int it = 0; it < kRefineR; ++it) {
      for (int i = 0; i < n; ++i) {
        double s = 0.;
#pragma unroll 4
        for (int j = 0; j < n; ++j) s += (double)jac[(long)(i * n + j) * ns] * x[j * kAT];
        tmp[i * ns] = r[i * ns] - (x[i * kAT] - hr0 * s);
      }
#pragma unroll 4
      for (int k = 0; k < n; ++k) d[k * kAT] = tmp[(long)perm[k * ns] * ns];
      lu_fwd_bwd<LUT>(d, lu, n, ns);
#pragma unroll 4
      for (int k = 0; k < n; ++k) x[k * kAT] += d[k * kAT];
    }
  }
}

__device__ __forceinline__ void copy_r(const double* __restrict__ s, double* __restrict__ d, int n, long ns) {
#pragma unroll 4
  for (int k = 0; k < n; ++k) d[k * ns] = s[k * ns];
}

// Buffers of the round scheme (all [field][ns], ns = capacity).
struct RoundBufs {
  long ns;
  double* sd;       // [ND_] scalar state
  int* si;          // [NI_] scalar state
  double* z;        // [8n] Nordsieck array
  double* v;        // [8n] predicted / corrected array
  double* b;
  double* f;
  double* f0;
  double* va;
  double* vb;
  double* eps;
  double* r;        // right-hand side of the current linear solve
  double* tmp;      // refinement residual
  float* jac;       // [n*n] finite-difference Jacobian
  void* lu;         // [n*n] factors (float or double)
  int* perm;        // [n] row permutation of the factors
  int* act0;        // active lists (round parity 0 / 1)
  int* act1;
  int* nact;        // [2] list lengths
};

}  // namespace

// ---------------------------------------------------------------------------
// init: gather, clip, renormalise (chemistry_DI.H:100-129), solver reset
// (MultiValueSolver.hpp:367-420); cells at or below tmin_chem finish here.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kAT) rounds_init_kernel(int NC, StepOptions o, StepArgs a, RoundBufs B) {
  const long ns = B.ns;
  const int n = NC + 1;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    B.nact[0] = (int)a.ncells;
    B.nact[1] = 0;
  }
  for (long cell = (long)blockIdx.x * blockDim.x + threadIdx.x; cell < a.ncells;
       cell += (long)gridDim.x * blockDim.x) {
    B.act0[cell] = (int)cell;
    int* si = B.si + cell;
    double* sd = B.sd + cell;
    const double Tc = a.T[cell];
    if (!(Tc > o.tmin_chem)) {
      double s = 0.;
      for (int i = 0; i < NC; ++i) s += a.Y[(long)i * a.ld + cell];
      for (int i = 0; i < NC; ++i) a.Y[(long)i * a.ld + cell] /= s;
      if (a.status) a.status[cell] = 0;
      if (a.nsteps) a.nsteps[cell] = 0;
      if (a.counters)
        for (int k = 0; k < NCNT; ++k) a.counters[(long)cell * NCNT + k] = 0;
      si[I_PHASE * ns] = PH_DONE;
      continue;
    }
    double* va = B.va + cell;
    double s = 0.;
    for (int i = 0; i < NC; ++i) {
      double yi = a.Y[(long)i * a.ld + cell];
      if (yi < 0.) yi = 0.;
      va[i * ns] = yi;
      s += yi;
    }
    for (int i = 0; i < NC; ++i) va[i * ns] /= s;
    va[NC * ns] = Tc;
    const double t0 = a.t0;
    sd[D_T * ns] = t0; sd[D_T0 * ns] = t0; sd[D_TOUT * ns] = t0; sd[D_TMESH * ns] = t0; sd[D_TSTAB * ns] = t0;
    sd[D_H * ns] = 0.; sd[D_HNEXT * ns] = 0.; sd[D_HNORD * ns] = 0.; sd[D_HSCALE * ns] = 0.;
    sd[D_HSCALEMAX * ns] = 1000.; sd[D_A24 * ns] = o.alfa2_4; sd[D_A25 * ns] = o.alfa2_5; sd[D_QR * ns] = 0.;
    sd[D_OLDCC * ns] = 0.; sd[D_HF * ns] = 0.; sd[D_HJ * ns] = 0.; sd[D_PENDHS * ns] = 0.; sd[D_HR0 * ns] = 0.;
    unsigned mij = 20u + 5u * (unsigned)(n - 3);
    if (mij > 50u && n < 80) mij = 50u;
    si[I_PHASE * ns] = PH_INIT; si[I_STATUS * ns] = 1; si[I_P * ns] = 1; si[I_ITORDER * ns] = 0;
    si[I_ORDNEXT * ns] = 1; si[I_MAXITJ * ns] = (int)mij; si[I_HSTAT * ns] = 1; si[I_OSTAT * ns] = 1;
    si[I_FACTORIZED * ns] = 0; si[I_JACCHANGE * ns] = 1; si[I_CONVOK * ns] = 1; si[I_NSTEPS * ns] = 0;
    si[I_ITCONV * ns] = 0; si[I_ITCONVRATE * ns] = 0; si[I_ITCONVFAIL * ns] = 0; si[I_ITERRFAIL * ns] = 0;
    si[I_NCFOM * ns] = 0; si[I_STEPLASTJ * ns] = 0; si[I_ITCONST * ns] = 0; si[I_ITMINORD * ns] = 0;
    si[I_FIXEDMIN * ns] = 0; si[I_NEWTONK * ns] = 0; si[I_JCOL * ns] = 0; si[I_MAXORD * ns] = o.maximum_order;
    for (int k = 0; k < NCNT; ++k) si[(I_CNT0 + k) * ns] = 0;
  }
}

// ---------------------------------------------------------------------------
// rhs: one thread per listed cell that requested an evaluation.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kRT) rounds_rhs_kernel(MechLayout Lp, const unsigned char* __restrict__ mech_gmem,
                                                          int energy, double P0, RoundBufs B, int par, int* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ MechLayout sL;
  if (threadIdx.x == 0) sL = Lp;
  if (blockIdx.x == 0 && threadIdx.x == 0) B.nact[par ^ 1] = 0;   // this round's compaction appends there
  if (!stage_bulk(smem, mech_gmem, Lp.bytes, &mbar, err)) return;
  const double* Md = (const double*)smem;
  const int* Mi = (const int*)(smem + (size_t)Lp.n_double * sizeof(double));
  double* scratch = (double*)(smem + ((Lp.bytes + 15u) & ~15u));
  const long ns = B.ns;
  const int nact = B.nact[par];
  const int* act = par ? B.act1 : B.act0;
  for (int idx = blockIdx.x * kRT + threadIdx.x; idx < nact; idx += gridDim.x * kRT) {
    const int cell = act[idx];
    int* si = B.si + cell;
    const int ph = si[I_PHASE * ns];
    if (!rhs_phase(ph)) continue;
    const double* src = B.va + cell;
    double* dst = B.f + cell;
    int pj = -1;
    double pval = 0.;
    if (ph == PH_PRED) {
      src = B.vb + cell;
      dst = B.f0 + cell;
    } else if (ph == PH_JAC) {
      src = B.vb + cell;
      pj = si[I_JCOL * ns];
      pval = src[(long)pj * ns] + B.sd[D_HJ * ns + cell];
    } else if (ph == PH_STAB_CONV || ph == PH_STAB_ERR) {
      src = B.z + cell;
    }
    const double QR = rhs_cell(&sL, Md, Mi, scratch, src, ns, pj, pval, dst, P0, energy);
    B.sd[D_QR * ns + cell] = QR;
    const int ck = (ph == PH_JAC) ? CNT_JAC_RHS : CNT_RHS;
    si[(I_CNT0 + ck) * ns] += 1;
  }
}

// ---------------------------------------------------------------------------
// advance: consume the RHS result (mode 0) or the fresh factorisation (mode 1)
// and run the cell's solver to its next request.
// ---------------------------------------------------------------------------
template <typename LUT>
__global__ void __launch_bounds__(kAT) rounds_advance_kernel(int NC, StepOptions o, StepArgs a, RoundBufs B, int par,
                                                              int mode) {
  extern __shared__ double sxd[];   // this thread's two solve vectors, element k at [k * kAT]
  const long ns = B.ns;
  const int n = NC + 1;
  double* const x = sxd + threadIdx.x;
  double* const dd = sxd + n * kAT + threadIdx.x;
  const int nact = B.nact[par];
  const int* act = par ? B.act1 : B.act0;
  const double yminT = o.y_min_T, ymaxT = o.y_max_T;
  for (int idx = blockIdx.x * kAT + threadIdx.x; idx < nact; idx += gridDim.x * kAT) {
    const int cell = act[idx];
    int* si = B.si + cell;
    double* sd = B.sd + cell;
    int phase = si[I_PHASE * ns];
    if (mode == 0 ? !rhs_phase(phase) : phase != PH_FACTORED) continue;
    double* const pz = B.z + cell;
    double* const pv = B.v + cell;
    double* const pb = B.b + cell;
    double* const pf = B.f + cell;
    double* const pf0 = B.f0 + cell;
    double* const pva = B.va + cell;
    double* const pvb = B.vb + cell;
    double* const peps = B.eps + cell;
    double* const pr = B.r + cell;
    double* const ptmp = B.tmp + cell;
    float* const pjac = B.jac + cell;
    const LUT* const plu = (const LUT*)B.lu + cell;
    const int* const pperm = B.perm + cell;
    // ---- the cell's scalar state ----
    double t = sd[D_T * ns];
    const double t0 = sd[D_T0 * ns];
    double tOut = sd[D_TOUT * ns], tInMeshPoint = sd[D_TMESH * ns];
    double tStabilize = sd[D_TSTAB * ns], h = sd[D_H * ns], hNextStep = sd[D_HNEXT * ns];
    double hNordsieck = sd[D_HNORD * ns], hScale = sd[D_HSCALE * ns], hScaleMax = sd[D_HSCALEMAX * ns];
    double alfa2_4 = sd[D_A24 * ns], alfa2_5 = sd[D_A25 * ns], oldCC = sd[D_OLDCC * ns];
    const double QR = sd[D_QR * ns];
    double hf = sd[D_HF * ns], hJ = sd[D_HJ * ns], pendHScale = sd[D_PENDHS * ns], hr0f = sd[D_HR0 * ns];
    int status = si[I_STATUS * ns];
    unsigned p = si[I_P * ns], iterOrder = si[I_ITORDER * ns], orderInNextStep = si[I_ORDNEXT * ns];
    const unsigned maxIterationsJacobian = si[I_MAXITJ * ns];
    int odeHStatus = si[I_HSTAT * ns], odeOrderStatus = si[I_OSTAT * ns], factorized = si[I_FACTORIZED * ns];
    int jacobianChange = si[I_JACCHANGE * ns], convOK = si[I_CONVOK * ns];
    unsigned numberOfSteps = si[I_NSTEPS * ns], iterConvergence = si[I_ITCONV * ns];
    unsigned iterConvergenceRate = si[I_ITCONVRATE * ns], iterConvergenceFailure = si[I_ITCONVFAIL * ns];
    unsigned iterErrorFailure = si[I_ITERRFAIL * ns], nConvFailOrderMax = si[I_NCFOM * ns];
    unsigned stepOfLastJacobian = si[I_STEPLASTJ * ns], iterConstSteps = si[I_ITCONST * ns];
    unsigned iterMinimumOrder = si[I_ITMINORD * ns];
    bool fixedOrderMin = si[I_FIXEDMIN * ns] != 0;
    unsigned newtonK = si[I_NEWTONK * ns];
    int jcol = si[I_JCOL * ns];
    unsigned maximum_order = si[I_MAXORD * ns];
    int cstep = 0, csolve = 0, cjac = 0, cfact = 0, cerr = 0, cconv = 0;

    enum : int { H_DEC = 0, H_CONST = 1, H_INC = 2 };
    enum : int { O_DEC = 0, O_CONST = 1, O_INC = 2 };
    auto alfa2 = [&](unsigned k) { return k == 4 ? alfa2_4 : (k == 5 ? alfa2_5 : .8); };
    auto Zp = [&](unsigned i) { return pz + (long)i * n * ns; };
    auto Vp = [&](unsigned i) { return pv + (long)i * n * ns; };

    enum : int { L_NONE, L_START_STEP, L_DRIVER_LOOP, L_JAC_COLUMN, L_AFTER_JAC, L_AFTER_FACT, L_NEWTON_TEST,
                 L_CORR_DONE, L_FINISH };
    int lab = L_NONE;
    switch (phase) {
      case PH_INIT: {
        // MultiValueSolver::Solve, first call (:445-469)
        bool illegal = false;
        for (int k = 0; k < n; ++k) {
          const double yk = pva[k * ns];
          if (yk < lo_b(k, NC, yminT) || yk > hi_b(k, NC, ymaxT)) illegal = true;
        }
        if (illegal) { status = -9; lab = L_FINISH; break; }
        set_eps_r(pva, peps, n, ns, o.atol, o.rtol);
        double lo, hi;
        if (t0 != 0.) { lo = 100. * kMachEpsDouble * fabs(t0); hi = fabs(t0); }
        else { lo = kMachEpsDouble; hi = 1.e-4; }
        double h0 = 0.5 / (wrms_r(pf, peps, n, ns) + kMachEpsFloat);
        if (h0 < lo) h0 = lo;
        if (h0 > hi) h0 = hi;
        const double dtc = a.dt ? a.dt[cell] : a.dt_scalar;
        tOut = t0 + dtc;
        h0 *= fabs(tOut - t0) / (tOut - t0);
        double* z1 = Zp(1);
        for (int k = 0; k < n; ++k) {
          pz[k * ns] = pva[k * ns];
          z1[k * ns] = pf[k * ns] * h0;
        }
        hNordsieck = h0; hNextStep = h0;
        status = 2;
        lab = L_START_STEP;
        break;
      }
      case PH_PRED: {
        // MethodGear::FindCorrection after f(vb) (:205-262)
        if (numberOfSteps >= stepOfLastJacobian + maxIterationsJacobian) jacobianChange = 1;
        if (jacobianChange) {
          stepOfLastJacobian = numberOfSteps;
          jacobianChange = 0;
          hf = 1.e+3 * kMachEpsDouble * fabs(h) * wrms_r(pf0, peps, n, ns) * double(n);
          if (hf < 1.e-10) hf = 1.;
          jcol = 0;
          lab = L_JAC_COLUMN;
          break;
        }
        lab = L_AFTER_JAC;
        break;
      }
      case PH_JAC: {
        const double hInv = 1. / hJ;
#pragma unroll 4
        for (int i = 0; i < n; ++i) pjac[(long)(i * n + jcol) * ns] = (float)(hInv * (pf[i * ns] - pf0[i * ns]));
        ++jcol;
        if (jcol < n) { lab = L_JAC_COLUMN; break; }
        ++cjac;
        factorized = 0;
        lab = L_AFTER_JAC;
        break;
      }
      case PH_NEWTON: {
        const double* v1 = Vp(1);
#pragma unroll 4
        for (int k = 0; k < n; ++k) pr[k * ns] = pf[k * ns] * h - v1[k * ns] - pb[k * ns];
        lin_solve_r<LUT>(x, dd, pr, plu, pperm, pjac, ptmp, hr0f, n, ns);
        ++csolve;
#pragma unroll 4
        for (int k = 0; k < n; ++k) pb[k * ns] += x[k * kAT];
        ++newtonK;
        if (newtonK > 4u) { convOK = 0; iterConvergence = 4; lab = L_CORR_DONE; }
        else lab = L_NEWTON_TEST;
        break;
      }
      case PH_STAB_CONV: {
        double* z1 = Zp(1);
        for (int k = 0; k < n; ++k) z1[k * ns] = pf[k * ns] * h;
        tStabilize = tInMeshPoint;
        if (numberOfSteps > stepOfLastJacobian + 5u) jacobianChange = 1;
        if (numberOfSteps != stepOfLastJacobian && iterConvergenceFailure == 50u) jacobianChange = 1;
        hNextStep *= pendHScale;
        lab = L_DRIVER_LOOP;
        break;
      }
      case PH_STAB_ERR: {
        double* z1 = Zp(1);
        for (int k = 0; k < n; ++k) z1[k * ns] = pf[k * ns] * h;
        tStabilize = tInMeshPoint;
        odeHStatus = H_DEC;
        hNextStep *= hScale;
        lab = L_DRIVER_LOOP;
        break;
      }
      case PH_FINAL:
        lab = L_FINISH;
        break;
      case PH_FACTORED:
        factorized = 1;
        ++cfact;
        lab = L_AFTER_FACT;
        break;
      default:
        status = -10;
        copy_r(pz, pva, n, ns);
        lab = L_FINISH;
        break;
    }

    // labels that need no RHS; a request or a finish is reached within a few hops
    for (int hop = 0; lab != L_NONE; ++hop) {
      if (hop >= 64) {
        status = -10;
        copy_r(pz, pva, n, ns);
        lab = L_FINISH;
      }
      switch (lab) {
        case L_START_STEP: {
          // MultiValueSolver::Solve loop (:532-560) + DriverStep prologue (:753-776)
          if (numberOfSteps >= (unsigned)o.max_steps) {
            status = -1;
            copy_r(pz, pva, n, ns);
            lab = L_FINISH;
            break;
          }
          set_eps_r(pz, peps, n, ns, o.atol, o.rtol);
          if (kMachEpsDouble * wrms_r(pz, peps, n, ns) > 1.) {
            status = -2;
            copy_r(pz, pva, n, ns);
            lab = L_FINISH;
            break;
          }
          tInMeshPoint = t;
          iterConvergenceFailure = 0; iterErrorFailure = 0; convOK = 1;
          if (odeOrderStatus != O_CONST || odeHStatus != H_CONST) iterOrder = 0;
          p = orderInNextStep;
          odeOrderStatus = O_CONST;
          hScaleMax = 2.;
          if (numberOfSteps < 10) hScaleMax = 1000.;
          else if (numberOfSteps > 10 && numberOfSteps < 20) hScaleMax = 10.;
          lab = L_DRIVER_LOOP;
          break;
        }
        case L_DRIVER_LOOP: {
          // DriverStep while(1) body up to FindCorrection (:778-820, :1212-1266)
          if (odeHStatus != H_CONST) {
            hScale = hNextStep / hNordsieck;
            rescale_z_r(pz, n, ns, p, hScale, NC, yminT, ymaxT);
            iterOrder = 0;
            odeHStatus = H_CONST;
          }
          h = hNextStep;
          hNordsieck = hNextStep;
          t = tInMeshPoint + h;
          if (t == tInMeshPoint) {
            status = -6;
            copy_r(pz, pva, n, ns);
            t = tInMeshPoint;
            lab = L_FINISH;
            break;
          }
          predict_r(pz, pv, pvb, peps, n, ns, p, NC, yminT, ymaxT);
          phase = PH_PRED;
          lab = L_NONE;
          break;
        }
        case L_JAC_COLUMN: {
          // KernelDense::NumericalJacobian, constrained branch: increment of column jcol
          const double yh = pvb[jcol * ns];
          const double ej = peps[jcol * ns];
          const double aa = fabs(yh), bb = fabs(1. / ej);
          hJ = sqrt(kMachEpsDouble) * (aa > bb ? aa : bb);
          hJ = fmax(hJ, hf / ej);
          hJ = fmax(hJ, sqrt(kTinyFloat));
          if (yh + hJ > hi_b(jcol, NC, ymaxT)) hJ = -hJ;
          phase = PH_JAC;
          lab = L_NONE;
          break;
        }
        case L_AFTER_JAC: {
          if (factorized && iterOrder == 0) factorized = 0;
          if (!factorized) {
            hr0f = h * c_gear_r.r[0][p - 1];
            phase = PH_FACT;
            lab = L_NONE;
            break;
          }
          lab = L_AFTER_FACT;
          break;
        }
        case L_AFTER_FACT: {
          const double* v1 = Vp(1);
#pragma unroll 4
          for (int k = 0; k < n; ++k) pr[k * ns] = pf0[k * ns] * h - v1[k * ns];
          lin_solve_r<LUT>(x, dd, pr, plu, pperm, pjac, ptmp, hr0f, n, ns);
          ++csolve;
#pragma unroll 4
          for (int k = 0; k < n; ++k) pb[k * ns] = x[k * kAT];
          newtonK = 1;
          lab = L_NEWTON_TEST;
          break;
        }
        case L_NEWTON_TEST: {
          const double r0 = c_gear_r.r[0][p - 1];
          double s2 = 0.;
#pragma unroll 4
          for (int k = 0; k < n; ++k) {
            const double c = x[k * kAT] * peps[k * ns];
            s2 += c * c;
          }
          const double cc = r0 * sqrt(s2 / double(n));
          if (cc < 1.) { convOK = 1; iterConvergence = newtonK; lab = L_CORR_DONE; break; }
          if (newtonK > 1 && cc > 2. * oldCC) { convOK = 0; iterConvergence = newtonK; lab = L_CORR_DONE; break; }
          oldCC = cc;
          const double* v0 = Vp(0);
#pragma unroll 4
          for (int k = 0; k < n; ++k) {
            double va = pb[k * ns] * r0 + v0[k * ns];
            const double lo = lo_b(k, NC, yminT), hi = hi_b(k, NC, ymaxT);
            if (va < lo) { va = lo; pb[k * ns] = (lo - pz[k * ns]) / r0; }
            if (va > hi) { va = hi; pb[k * ns] = (hi - pz[k * ns]) / r0; }
            pva[k * ns] = va;
          }
          phase = PH_NEWTON;
          lab = L_NONE;
          break;
        }
        case L_CORR_DONE: {
          if (!convOK) {
            // DriverStep convergence-failure branch (:822-847) + recovery (MethodGear.hpp:343-423)
            iterConvergenceFailure++;
            ++cconv;
            if (iterConvergenceFailure >= 50u || fabs(h) <= 0.) {
              status = iterConvergenceFailure >= 50u ? -5 : -6;
              copy_r(pz, pva, n, ns);
              t = tInMeshPoint;
              lab = L_FINISH;
              break;
            }
            double hs = 0.25;
            if (numberOfSteps < 10) hs = 0.1;
            hs = fmax(hs, 0. / fabs(h));
            odeHStatus = H_DEC;
            if (p > 1u) { p -= 1; odeOrderStatus = O_DEC; }
            alfa2_4 -= 0.01;
            alfa2_5 -= 0.02;
            if (alfa2_4 < 0.) { alfa2_4 = 0.; maximum_order = 3; if (p > 3) { p = 3; odeOrderStatus = O_DEC; } }
            if (alfa2_5 < 0.) { alfa2_5 = 0.; maximum_order = 4; if (p > 4) { p = 4; odeOrderStatus = O_DEC; } }
            hScale = hs;
            pendHScale = hs;
            if (numberOfSteps > 5) {
              nConvFailOrderMax++;
              if (nConvFailOrderMax % 5 == 0 && p != 1u) { p = 1; odeOrderStatus = O_DEC; }
              if (nConvFailOrderMax % 10 == 0 && tStabilize != tInMeshPoint) {
                phase = PH_STAB_CONV;
                lab = L_NONE;
                break;
              }
            }
            if (numberOfSteps > stepOfLastJacobian + 5u) jacobianChange = 1;
            if (numberOfSteps != stepOfLastJacobian && iterConvergenceFailure == 50u) jacobianChange = 1;
            hNextStep *= hs;
            lab = L_DRIVER_LOOP;
            break;
          }
          // MultiValueStep tail (:1271-1327)
          {
            const double r0 = c_gear_r.r[0][p - 1];
            double* v0 = Vp(0);
            double* v1 = Vp(1);
            for (int k = 0; k < n; ++k) {
              const double lo = lo_b(k, NC, yminT), hi = hi_b(k, NC, ymaxT);
              double b = pb[k * ns];
              const double va = b * r0;
              double x0 = v0[k * ns];
              const double x1 = v1[k * ns];
              const double z0 = pz[k * ns];
              if (x0 + va < lo) { b = lo - z0 - x1; x0 = lo - va; if (x0 < lo) x0 = lo; }
              if (x0 + va > hi) { b = hi - z0 - x1; x0 = hi - va; if (x0 > hi) x0 = hi; }
              v0[k * ns] = x0 + va;
              v1[k * ns] = x1 + b;
              pb[k * ns] = b;
            }
            for (unsigned i = 2; i <= p; ++i) {
              const double ri = c_gear_r.r[i][p - 1];
              double* vi = Vp(i);
#pragma unroll 4
              for (int k = 0; k < n; ++k) vi[k * ns] += pb[k * ns] * ri;
            }
            {
              double* vp1 = Vp(p + 1);
              const double* vpp = Vp(p);
              const double* zpp = Zp(p);
              for (int k = 0; k < n; ++k) vp1[k * ns] = (vpp[k * ns] - zpp[k * ns]) / (double(p) + 1.);
            }
            if (iterOrder >= p) {
              double* vp2 = Vp(p + 2);
              const double* vp1 = Vp(p + 1);
              const double* zp1 = Zp(p + 1);
              for (int k = 0; k < n; ++k) vp2[k * ns] = (vp1[k * ns] - zp1[k * ns]) / (double(p) + 2.);
            }
          }
          // error test (:876-962)
          double hCur = c_gear_r.Ep[p] * wrms_r(Vp(p + 1), peps, n, ns);
          if (hCur > 1.) {
            iterErrorFailure++;
            ++cerr;
            if (iterErrorFailure >= 50u || fabs(h) <= 0.) {
              status = iterErrorFailure >= 50u ? -4 : -6;
              copy_r(pz, pva, n, ns);
              t = tInMeshPoint;
              lab = L_FINISH;
              break;
            }
            hScaleMax = 1.;
            hCur = 0.8 * pow(1. / hCur, 1. / double(p + 1));
            hScale = hCur;
            if (p > 1u) {
              double hMinus = c_gear_r.Ep[p - 1] * wrms_r(Vp(p), peps, n, ns);
              hMinus = 1. / (hMinus + kMachEpsFloat);
              hMinus = 0.8 * pow(hMinus, 1. / double(p));
              if (hMinus > hCur) { hScale = hMinus; p -= 1; odeOrderStatus = O_DEC; }
            }
            hScale = fmin(hScale, 0.5);
            hScale = fmax(hScale, 0. / fabs(h));
            hScale = fmax(hScale, 1.e-3);
            if (p == 1u && hScale < 0.1 && numberOfSteps > 10 && tInMeshPoint != tStabilize) {
              phase = PH_STAB_ERR;
              lab = L_NONE;
              break;
            }
            odeHStatus = H_DEC;
            hNextStep *= hScale;
            lab = L_DRIVER_LOOP;
            break;
          }
          // accepted step (:963-1037)
          hNordsieck = h; hNextStep = h;
          orderInNextStep = p; odeOrderStatus = O_CONST; odeHStatus = H_CONST;
          {
            // MethodGear::ConvergenceRate (:425-516) with the stored Jacobian
            if (iterErrorFailure > 0 || iterConvergenceFailure > 0) iterConvergenceRate = 0;
            if (iterConvergence > 1) {
              const double* v0 = Vp(0);
              const double* v1 = Vp(1);
              const double* z1 = Zp(1);
#pragma unroll 4
              for (int j = 0; j < n; ++j) x[j * kAT] = v0[j * ns] - pz[j * ns];
              double normd = 0., normf = 0.;
              for (int i = 0; i < n; ++i) {
                double s = 0.;
#pragma unroll 4
                for (int j = 0; j < n; ++j) s += (double)pjac[(long)(i * n + j) * ns] * x[j * kAT];
                const double va = v1[i * ns] - (s * h + z1[i * ns]);
                normd += fabs(va);
                normf += fabs(v1[i * ns]);
              }
              if (normd > 3. * normf + .1 && iterConvergence > 2) {
                if (numberOfSteps > stepOfLastJacobian + 5u) jacobianChange = 1;
                hScale = 0.5; odeHStatus = H_DEC; hNextStep = h * hScale;
                if (p > 1) { orderInNextStep = p - 1; odeOrderStatus = O_DEC; }
                iterConvergenceRate = 0; iterConvergenceFailure = 1;
              } else if (normd > normf + 0.1) {
                iterConvergenceRate++;
                if (iterConvergenceRate >= 5) {
                  hScale = 0.8; odeHStatus = H_DEC; hNextStep = h * hScale;
                  iterConvergenceRate = 0; iterConvergenceFailure = 1;
                }
                if (numberOfSteps > stepOfLastJacobian + 5u && iterConvergence > 2) {
                  jacobianChange = 1;
                  iterConvergenceRate = 0; iterConvergenceFailure = 1;
                }
              }
            }
          }
          if (iterErrorFailure > 0 || iterConvergenceFailure > 0) {
            iterErrorFailure = 0; iterConvergenceFailure = 0;
          } else {
            iterOrder++;
            if (iterOrder > p + 1) {
              // NewOrderNewH (:1042-1210)
              double hMinus = 0., hC = 0., hPlus = 0., alfa1 = 0., alfa3 = 0.;
              if (p > 1u && odeOrderStatus != O_INC) {
                hMinus = c_gear_r.Ep[p - 1] * wrms_r(Vp(p), peps, n, ns) + kMachEpsFloat;
                hMinus = 1. / hMinus;
                alfa1 = alfa2(p - 1) - .05;
                hMinus = alfa1 * pow(hMinus, 1. / double(p));
              }
              hC = c_gear_r.Ep[p] * wrms_r(Vp(p + 1), peps, n, ns) + kMachEpsFloat;
              hC = 1. / hC;
              hC = alfa2(p) * pow(hC, 1. / double(p + 1));
              if (p < maximum_order && odeOrderStatus != O_DEC) {
                hPlus = c_gear_r.Ep[p + 1] * wrms_r(Vp(p + 2), peps, n, ns) + kMachEpsFloat;
                hPlus = 1. / hPlus;
                alfa3 = alfa2(p + 1) - .25;
                hPlus = alfa3 * pow(hPlus, 1. / double(p + 2));
              }
              if (hMinus > hC && hMinus > hPlus) {
                hScale = (.75 / alfa1) * hMinus; orderInNextStep = p - 1; odeOrderStatus = O_DEC;
              } else if (hC > hMinus && hC > hPlus) {
                hScale = (.75 / alfa2(p)) * hC; orderInNextStep = p; odeOrderStatus = O_CONST;
              } else {
                hScale = (.75 / alfa3) * hPlus; orderInNextStep = p + 1; odeOrderStatus = O_INC;
              }
              if (fixedOrderMin) {
                iterMinimumOrder++;
                if (iterMinimumOrder < 2000) {
                  hScale = (.75 / alfa2(p)) * hC; orderInNextStep = p; odeOrderStatus = O_CONST;
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
          }
          for (unsigned i = 0; i <= p + 2; ++i) copy_r(Vp(i), Zp(i), n, ns);
#pragma unroll 4
          for (int k = 0; k < n; ++k) {
            double z0 = pz[k * ns];
            const double lo = lo_b(k, NC, yminT), hi = hi_b(k, NC, ymaxT);
            if (z0 < lo) z0 = lo;
            if (z0 > hi) z0 = hi;
            pz[k * ns] = z0;
          }
          numberOfSteps++;
          ++cstep;
          if (tOut == t) {
            copy_r(pz, pva, n, ns);
            lab = L_FINISH;
            break;
          }
          if (tOut < t) {
            // Interpolation (:687-706); the RHS at tOut then sets QR (:599-611)
            const double hp = (tOut - t) / hNordsieck;
            for (int k = 0; k < n; ++k) {
              double yv = pz[k * ns];
              if (hp != 0.) {
                double hr = 1.;
                for (unsigned i = 1; i <= p; ++i) { hr *= hp; yv += Zp(i)[k * ns] * hr; }
                const double lo = lo_b(k, NC, yminT), hi = hi_b(k, NC, ymaxT);
                if (yv < lo) yv = lo;
                if (yv > hi) yv = hi;
              }
              pva[k * ns] = yv;
            }
            phase = PH_FINAL;
            lab = L_NONE;
            break;
          }
          lab = L_START_STEP;
          break;
        }
        case L_FINISH: {
          // utilities.H:153-200 and the scatter of chemistry_DI.H:221-235
          double s = 0.;
          for (int i = 0; i < NC; ++i) s += pva[i * ns];
          for (int i = 0; i < NC; ++i) a.Y[(long)i * a.ld + cell] = pva[i * ns] / s;
          if (o.energy) a.T[cell] = pva[NC * ns];
          if (a.Q) a.Q[cell] = QR;
          if (a.status) a.status[cell] = status;
          if (a.nsteps) a.nsteps[cell] = (int)numberOfSteps;
          phase = PH_DONE;
          lab = L_NONE;
          break;
        }
        default:
          lab = L_NONE;
          break;
      }
    }
    // ---- store the cell's scalar state ----
    sd[D_T * ns] = t; sd[D_TOUT * ns] = tOut; sd[D_TMESH * ns] = tInMeshPoint; sd[D_TSTAB * ns] = tStabilize;
    sd[D_H * ns] = h; sd[D_HNEXT * ns] = hNextStep; sd[D_HNORD * ns] = hNordsieck; sd[D_HSCALE * ns] = hScale;
    sd[D_HSCALEMAX * ns] = hScaleMax; sd[D_A24 * ns] = alfa2_4; sd[D_A25 * ns] = alfa2_5;
    sd[D_OLDCC * ns] = oldCC; sd[D_HF * ns] = hf; sd[D_HJ * ns] = hJ; sd[D_PENDHS * ns] = pendHScale;
    sd[D_HR0 * ns] = hr0f;
    si[I_PHASE * ns] = phase; si[I_STATUS * ns] = status; si[I_P * ns] = (int)p; si[I_ITORDER * ns] = (int)iterOrder;
    si[I_ORDNEXT * ns] = (int)orderInNextStep; si[I_HSTAT * ns] = odeHStatus; si[I_OSTAT * ns] = odeOrderStatus;
    si[I_FACTORIZED * ns] = factorized; si[I_JACCHANGE * ns] = jacobianChange; si[I_CONVOK * ns] = convOK;
    si[I_NSTEPS * ns] = (int)numberOfSteps; si[I_ITCONV * ns] = (int)iterConvergence;
    si[I_ITCONVRATE * ns] = (int)iterConvergenceRate; si[I_ITCONVFAIL * ns] = (int)iterConvergenceFailure;
    si[I_ITERRFAIL * ns] = (int)iterErrorFailure; si[I_NCFOM * ns] = (int)nConvFailOrderMax;
    si[I_STEPLASTJ * ns] = (int)stepOfLastJacobian; si[I_ITCONST * ns] = (int)iterConstSteps;
    si[I_ITMINORD * ns] = (int)iterMinimumOrder; si[I_FIXEDMIN * ns] = fixedOrderMin ? 1 : 0;
    si[I_NEWTONK * ns] = (int)newtonK; si[I_JCOL * ns] = jcol; si[I_MAXORD * ns] = (int)maximum_order;
    int c8[NCNT];
#pragma unroll
    for (int k = 0; k < NCNT; ++k) c8[k] = si[(I_CNT0 + k) * ns];
    c8[CNT_STEPS] += cstep; c8[CNT_JAC] += cjac; c8[CNT_FACT] += cfact; c8[CNT_SOLVE] += csolve;
    c8[CNT_ERRFAIL] += cerr; c8[CNT_CONVFAIL] += cconv;
#pragma unroll
    for (int k = 0; k < NCNT; ++k) si[(I_CNT0 + k) * ns] = c8[k];
    if (phase == PH_DONE && a.counters)
      for (int k = 0; k < NCNT; ++k) a.counters[(long)cell * NCNT + k] = c8[k];
  }
}

// ---------------------------------------------------------------------------
// factor: one warp per cell that requested a factorisation.  G = I - hr0 J
// (built in FP64, stored as LUT), partial pivoting on the largest magnitude,
// first occurrence (KernelDense LU), rows = lanes, matrix in shared memory.
// The factors are stored as P G = L U with perm[k] = row of G in position k.
// ---------------------------------------------------------------------------
template <typename LUT>
__global__ void __launch_bounds__(kFW * 32) rounds_factor_kernel(int NC, RoundBufs B, int par) {
  extern __shared__ __align__(16) unsigned char fsm[];
  const long ns = B.ns;
  const int n = NC + 1, ld = n + 1;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  LUT* G = (LUT*)fsm + (size_t)w * n * ld;
  int* rowof = (int*)((LUT*)fsm + (size_t)kFW * n * ld) + w * 32;
  const int nact = B.nact[par];
  const int* act = par ? B.act1 : B.act0;
  const int nwarps = gridDim.x * kFW;
  for (int base = (blockIdx.x * kFW + w) * 32; base < nact; base += nwarps * 32) {
    const int idx = base + lane;
    const int mycell = idx < nact ? act[idx] : 0;
    const bool want = idx < nact && B.si[I_PHASE * ns + mycell] == PH_FACT;
    unsigned m = __ballot_sync(kFull, want);
    while (m) {
      const int q = __ffs(m) - 1;
      m &= m - 1;
      const int cell = __shfl_sync(kFull, mycell, q);
      const double hr0 = B.sd[D_HR0 * ns + cell];
      const float* J = B.jac + cell;
      if (lane < n) {
        for (int j = 0; j < n; ++j) {
          double g = -hr0 * (double)J[(long)(lane * n + j) * ns];
          if (j == lane) g += 1.;
          G[lane * ld + j] = (LUT)g;
        }
      }
      rowof[lane] = lane;   // rowof[k]: row of G now in position k
      __syncwarp();
      for (int k = 0; k < n; ++k) {
        LUT v = (lane >= k && lane < n) ? (LUT)fabs((double)G[lane * ld + k]) : (LUT)-1;
        int r = lane;
        for (int off = 16; off > 0; off >>= 1) {
          const LUT ov = __shfl_xor_sync(kFull, v, off);
          const int orr = __shfl_xor_sync(kFull, r, off);
          if (ov > v || (ov == v && orr < r)) { v = ov; r = orr; }
        }
        // one pivot for the whole warp; a NaN column cannot send it outside rows k..n-1
        r = __shfl_sync(kFull, r, 0);
        if (r < k || r >= n) r = k;
        if (r != k) {
          if (lane < n) {
            const LUT tmp = G[k * ld + lane];
            G[k * ld + lane] = G[r * ld + lane];
            G[r * ld + lane] = tmp;
          }
          if (lane == 0) {
            const int t = rowof[k];
            rowof[k] = rowof[r];
            rowof[r] = t;
          }
        }
        __syncwarp();
        const LUT d = G[k * ld + k];
        if (lane > k && lane < n) {
          LUT l = G[lane * ld + k];
          if (d != (LUT)0) l /= d;
          G[lane * ld + k] = l;
          for (int j = k + 1; j < n; ++j) G[lane * ld + j] -= l * G[k * ld + j];
        }
        __syncwarp();
      }
      LUT* lu = (LUT*)B.lu + cell;
      if (lane < n) {
        for (int j = 0; j < n; ++j) lu[(long)(lane * n + j) * ns] = G[lane * ld + j];
        B.perm[(long)lane * ns + cell] = rowof[lane];
      }
      if (lane == 0) B.si[I_PHASE * ns + cell] = PH_FACTORED;
      __syncwarp();
    }
  }
}

// ---------------------------------------------------------------------------
// compact: cells still integrating form the next list (warp-aggregated append).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kCT) rounds_compact_kernel(RoundBufs B, int par) {
  const long ns = B.ns;
  const int nact = B.nact[par];
  const int* in = par ? B.act1 : B.act0;
  int* out = par ? B.act0 : B.act1;
  int* cnt = B.nact + (par ^ 1);
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * kCT + threadIdx.x) >> 5;
  const int nw = gridDim.x * (kCT / 32);
  for (int base = gw * 32; base < nact; base += nw * 32) {
    const int idx = base + lane;
    const int cell = idx < nact ? in[idx] : 0;
    const bool alive = idx < nact && B.si[I_PHASE * ns + cell] != PH_DONE;
    const unsigned m = __ballot_sync(kFull, alive);
    int off = 0;
    if (lane == 0 && m) off = atomicAdd(cnt, __popc(m));
    off = __shfl_sync(kFull, off, 0);
    if (alive) out[off + __popc(m & ((1u << lane) - 1u))] = cell;
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

RoundBufs carve(const MechLayout& L, void* base, long ns, bool lu64) {
  const int n = L.nc + 1;
  RoundBufs B{};
  B.ns = ns;
  char* p = (char*)base;
  auto take = [&](size_t bytes) {
    char* r = p;
    p += (bytes + 255) & ~(size_t)255;
    return (void*)r;
  };
  B.sd = (double*)take(sizeof(double) * ND_ * ns);
  B.si = (int*)take(sizeof(int) * NI_ * ns);
  B.z = (double*)take(sizeof(double) * 8 * n * ns);
  B.v = (double*)take(sizeof(double) * 8 * n * ns);
  B.b = (double*)take(sizeof(double) * n * ns);
  B.f = (double*)take(sizeof(double) * n * ns);
  B.f0 = (double*)take(sizeof(double) * n * ns);
  B.va = (double*)take(sizeof(double) * n * ns);
  B.vb = (double*)take(sizeof(double) * n * ns);
  B.eps = (double*)take(sizeof(double) * n * ns);
  B.r = (double*)take(sizeof(double) * n * ns);
  B.tmp = (double*)take(sizeof(double) * n * ns);
  B.jac = (float*)take(sizeof(float) * n * n * ns);
  B.lu = take((lu64 ? sizeof(double) : sizeof(float)) * n * n * ns);
  B.perm = (int*)take(sizeof(int) * n * ns);
  B.act0 = (int*)take(sizeof(int) * ns);
  B.act1 = (int*)take(sizeof(int) * ns);
  B.nact = (int*)take(sizeof(int) * 2);
  return B;
}

// One round's kernels for a factor type.
template <typename LUT>
struct RoundKernels {
  static cudaError_t prepare(size_t as, size_t fs, int* adv_bps, int* fac_bps) {
    cudaError_t e = cudaFuncSetAttribute(rounds_factor_kernel<LUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)fs);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(rounds_advance_kernel<LUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)as);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(adv_bps, rounds_advance_kernel<LUT>, kAT, as);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(fac_bps, rounds_factor_kernel<LUT>, kFW * 32, fs);
  }
  static void launch(const RoundsPlan& P, const MechLayout& L, const unsigned char* mech, const StepOptions& o,
                     const StepArgs& a, const RoundBufs& B, int par, int* err, cudaStream_t s) {
    rounds_rhs_kernel<<<P.g_rhs, kRT, P.rhs_smem, s>>>(L, mech, o.energy, a.p, B, par, err);
    rounds_advance_kernel<LUT><<<P.g_adv, kAT, P.adv_smem, s>>>(L.nc, o, a, B, par, 0);
    rounds_factor_kernel<LUT><<<P.g_fac, kFW * 32, P.fac_smem, s>>>(L.nc, B, par);
    rounds_advance_kernel<LUT><<<P.g_adv, kAT, P.adv_smem, s>>>(L.nc, o, a, B, par, 1);
    rounds_compact_kernel<<<P.g_cmp, kCT, 0, s>>>(B, par);
  }
};

}  // namespace

size_t rounds_bytes(const MechLayout& L, long ns, bool lu64) {
  const int n = L.nc + 1;
  auto r = [](size_t b) { return (b + 255) & ~(size_t)255; };
  return r(sizeof(double) * ND_ * ns) + r(sizeof(int) * NI_ * ns) + 2 * r(sizeof(double) * 8 * n * ns) +
         10 * r(sizeof(double) * n * ns) + r(sizeof(float) * n * n * ns) +
         r((lu64 ? sizeof(double) : sizeof(float)) * n * n * ns) + r(sizeof(int) * n * ns) +
         2 * r(sizeof(int) * ns) + r(sizeof(int) * 2);
}

cudaError_t upload_gear_rounds(const GearConsts& gc) { return cudaMemcpyToSymbol(c_gear_r, &gc, sizeof(GearConsts)); }

cudaError_t rounds_prepare(const MechLayout& L, bool lu64, int sm_count, RoundsPlan* P) {
  const int n = L.nc + 1;
  if (n > 32) return cudaErrorInvalidValue;
  *P = RoundsPlan{};
  P->lu64 = lu64;
  P->rhs_smem = ((L.bytes + 15u) & ~15u) + (size_t)4 * L.nc * kRT * sizeof(double);
  P->adv_smem = (size_t)2 * n * kAT * sizeof(double);
  P->fac_smem = (size_t)kFW * n * (n + 1) * (lu64 ? sizeof(double) : sizeof(float)) + kFW * 32 * sizeof(int);
  cudaError_t e = cudaFuncSetAttribute(rounds_rhs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)P->rhs_smem);
  if (e != cudaSuccess) return e;
  int rhs_bps = 0, adv_bps = 0, fac_bps = 0, cmp_bps = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&rhs_bps, rounds_rhs_kernel, kRT, P->rhs_smem);
  if (e != cudaSuccess) return e;
  if (lu64) e = RoundKernels<double>::prepare(P->adv_smem, P->fac_smem, &adv_bps, &fac_bps);
  else e = RoundKernels<float>::prepare(P->adv_smem, P->fac_smem, &adv_bps, &fac_bps);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cmp_bps, rounds_compact_kernel, kCT, 0);
  if (e != cudaSuccess) return e;
  if (rhs_bps <= 0 || adv_bps <= 0 || fac_bps <= 0 || cmp_bps <= 0) return cudaErrorInvalidConfiguration;
  // persistent grids: every kernel fills the GPU once and strides over the list
  P->g_rhs = (unsigned)(sm_count * rhs_bps);
  P->g_adv = (unsigned)(sm_count * adv_bps);
  P->g_fac = (unsigned)(sm_count * fac_bps);
  P->g_cmp = (unsigned)(sm_count * cmp_bps);
  P->g_init = (unsigned)(sm_count * 8);
  return cudaSuccess;
}

cudaError_t launch_rounds(const RoundsPlan& P, const MechLayout& L, const unsigned char* mech_gmem,
                          const StepOptions& o, const StepArgs& a, void* state, long ns, int* nact_host,
                          long max_rounds, int* err, cudaStream_t stream, long long* launches) {
  // nact_host: two pinned ints (list length, error flags); launches: kernels enqueued (added to)
  const int n = L.nc + 1;
  if (n > 32 || a.ncells > ns || a.ncells <= 0) return cudaErrorInvalidValue;
  const RoundBufs B = carve(L, state, ns, P.lu64);
  rounds_init_kernel<<<P.g_init, kAT, 0, stream>>>(L.nc, o, a, B);
  *launches += 1;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int kBatch = 8;   // rounds between host checks of the list length
  int par = 0;
  for (long round = 0; round < max_rounds; round += kBatch) {
    for (int r = 0; r < kBatch; ++r) {
      if (P.lu64) RoundKernels<double>::launch(P, L, mech_gmem, o, a, B, par, err, stream);
      else RoundKernels<float>::launch(P, L, mech_gmem, o, a, B, par, err, stream);
      *launches += 5;
      par ^= 1;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(nact_host, B.nact + par, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(nact_host + 1, err, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return e;
    if (nact_host[0] == 0) return cudaSuccess;
    if (nact_host[1] != 0) return cudaErrorLaunchTimeout;   // a kernel raised a flag: stop, the caller reports it
  }
  return cudaErrorLaunchTimeout;
}

}  // namespace lsg
