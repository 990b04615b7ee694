// Warp-per-cell FP64 reaction step for mechanisms with NC+1 <= 32 equations.
//
// One warp integrates one cell.  Lane l owns ODE component l (species mass
// fraction l, lane NC owns T); reaction-parallel work (rate constants,
// products of concentrations) is spread over the 32 lanes.  Every quantity the
// reference accumulates sequentially (mixture sums, WRMS norms, L1 norms,
// formation rates, reaction enthalpies) is accumulated in the same order here
// (seq_sum), so with FMA contraction disabled this path reproduces the CPU
// algorithm operation for operation; the remaining differences come from the
// device exp/log/pow, which agree with the host's to about one ulp.
//
// Algorithm followed (paths relative to solvers/openSMOKEpp4laminarSMOKE):
//   RHS        solvers/laminarSMOKE/unsteady/BatchReactorHomogeneousConstantPressure.H:175-223
//   thermo     maps/ThermodynamicsMap_CHEMKIN.hpp:429-520
//   kinetics   maps/KineticsMap_CHEMKIN.hpp:271-297, 1181-1398, 1496-1550, 1683-1768, 1956-1964
//   stoich.    maps/StoichiometricMap.hpp:512-598, 656-729, 916-1001
//   BDF        math/native-ode-solvers/MultiValueSolver.hpp:367-1328
//   Gear       math/native-ode-solvers/MethodGear.hpp:79-536
//   dense      math/native-ode-solvers/KernelDense.hpp:90-245
#pragma once
#include "lsg_common.cuh"
#include "lsg_kernels.h"

namespace lsg {

// One copy per translation unit; the host uploads it with cudaMemcpyToSymbol.
static __constant__ GearConsts c_gear;

// Per-warp shared-memory workspace (all arrays lane- or index-addressed).
struct WarpWS {
  double* Z;      // [8][32] Nordsieck array z_
  double* V;      // [8][32] v_
  double* J;      // [n][n+1] Jacobian, row major
  double* G;      // [n][n+1] LU factors of G = I - h r0 J
  double* C;      // [32] concentrations
  double* H;      // [32] h/RT
  double* S;      // [32] s/R
  double* KARR;   // [NR] forward Arrhenius constants (cache)
  double* UKEQ;   // [NR] 1/Keq (thermo reversible) or k_rev (explicit)
  double* NET;    // [NR] net rates
  double* KINF;   // [NFO] k_inf (cache)
  double* LOGF;   // [NFO] log10 Fcent (Troe) / SRI factor (cache)
  int* PIV;       // [32]
  double* SC;     // [6] scalars: cached kinetic T, QR of the last call, P0, energy flag, rho0 (> 0: constant volume)
  unsigned char* DROP;   // [NR] DRG-reduced step only (drg_ws_doubles): 1 for a reaction the analysis dropped
};

__host__ __device__ inline int warp_ws_doubles(const MechLayout& L) {
  const int n = L.nc + 1;
  auto even = [](int x) { return (x + 1) & ~1; };
  return 8 * 32 * 2 + even(n * (n + 1)) * 2 + 32 * 3 + even(L.nr) * 3 + even(L.n_fo > 0 ? L.n_fo : 1) * 2 + 16 + 6;
}

// The DRG kernel's per-warp workspace: the above and the dropped-reaction mask after it.
__host__ __device__ inline int drg_ws_doubles(const MechLayout& L) { return warp_ws_doubles(L) + (L.nr + 7) / 8 + 1; }

__device__ __forceinline__ WarpWS carve_ws(double* base, const MechLayout& L) {
  const int n = L.nc + 1;
  auto even = [](int x) { return (x + 1) & ~1; };
  WarpWS w;
  double* p = base;
  w.Z = p; p += 8 * 32;
  w.V = p; p += 8 * 32;
  w.J = p; p += even(n * (n + 1));
  w.G = p; p += even(n * (n + 1));
  w.C = p; p += 32;
  w.H = p; p += 32;
  w.S = p; p += 32;
  w.KARR = p; p += even(L.nr);
  w.UKEQ = p; p += even(L.nr);
  w.NET = p; p += even(L.nr);
  w.KINF = p; p += even(L.n_fo > 0 ? L.n_fo : 1);
  w.LOGF = p; p += even(L.n_fo > 0 ? L.n_fo : 1);
  w.PIV = (int*)p; p += 16;
  w.SC = p; p += 6;
  w.DROP = (unsigned char*)p;
  return w;
}

__device__ __forceinline__ double contrib(double nu, double v) {
  if (nu == 1.) return v;
  if (nu == 2.) return v + v;
  if (nu == 3.) return v + v + v;
  if (nu == 0.5) return 0.5 * v;
  return nu * v;
}

__device__ __forceinline__ double conc_factor(double nu, double c1) {
  if (nu == 1.) return c1;
  if (nu == 2.) return c1 * c1;
  if (nu == 3.) return c1 * c1 * c1;
  if (nu == 0.5) return sqrt(c1);
  return pow(c1, nu);
}

// ---------------------------------------------------------------------------
// Right-hand side f(y), warp cooperative.  yl: this lane's component.
// kT: cached temperature of the kinetic constants (the reference's T_old test).
// ---------------------------------------------------------------------------
// One out-of-line body (every caller shares it, keeping the kernel's
// instruction footprint small).  L points to the layout in shared memory,
// ws to this warp's workspace; the cached kinetic temperature, the last QR,
// P0 and the energy flag live in ws's scalar slots.
template <bool kDrg = false>
__device__ __noinline__ double rhs_warp(const MechLayout* __restrict__ Lp, const double* __restrict__ Md,
                                        const int* __restrict__ Mi, double* __restrict__ ws, double yl, double T) {
  const MechLayout& L = *Lp;
  const MechView M{Md, Mi};
  WarpWS W = carve_ws(ws, L);
  const double P0 = W.SC[2];
  const bool energy = W.SC[3] != 0.;
  const double rho0 = W.SC[4];   // constant volume when > 0 (BatchReactorHomogeneousConstantVolume.H:148-199)
  const bool cv = rho0 > 0.;
  const int lane = threadIdx.x & 31;
  const int NC = L.nc, NR = L.nr;
  const double* MW = M.D(L.mw);
  const double mwl = lane < NC ? MW[lane] : 1.;
  // mole fractions, concentrations, density
  const double q = lane < NC ? yl / mwl : 0.;
  const double u = seq_sum(q, NC);
  const double MWmix = 1. / u;
  double xl = 0.;
  if (lane < NC) { xl = MWmix * yl; xl = xl / mwl; }
  const double cTot = cv ? rho0 / MWmix : P0 / kRgas / T;
  const double cl = cTot * xl;
  const double rho = cv ? rho0 : cTot * MWmix;
  const double* TM = M.D(L.t_mid);
  const double T2 = T * T, T3 = T2 * T, T4 = T3 * T, uT = 1. / T;
  double hl = 0.;
  if (lane < NC) {
    const double* HT = M.D(L.dh_ht) + 6 * lane;
    const double* LT = M.D(L.dh_lt) + 6 * lane;
    const double* A = T > TM[lane] ? HT : LT;
    hl = A[0] + T * A[1] + T2 * A[2] + T3 * A[3] + T4 * A[4] + uT * A[5];
    W.C[lane] = cl;
    W.H[lane] = hl;
  }
  const double T_old = W.SC[0];
  const bool recalc = fabs(T - T_old) / T > 0.;
  __syncwarp();
  if (lane == 0) W.SC[0] = T;
  if (recalc && lane < NC) {
    const double logT = log(T);
    const double* HT = M.D(L.ds_ht) + 6 * lane;
    const double* LT = M.D(L.ds_lt) + 6 * lane;
    const double* A = T > TM[lane] ? HT : LT;
    W.S[lane] = A[0] * logT + T * A[1] + T2 * A[2] + T3 * A[3] + T4 * A[4] + A[5];
  }
  __syncwarp();
  if (recalc) {
    const double logT = log(T);
    const double Patm_over_RT = 101325. / kRgas / T;
    const double lP = log(Patm_over_RT);
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
    for (int j = lane; j < NR; j += 32) {
      double k = exp(lnA[j] + beta[j] * logT - eor[j] * uT);
      if (sgn[j] < 0) k *= -1.;
      W.KARR[j] = k;
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
            dh -= contrib(rnu[a], W.H[sa]);
            ds -= contrib(rnu[a], W.S[sa]);
            ++a;
          } else {
            dh += contrib(pnu[b], W.H[sb]);
            ds += contrib(pnu[b], W.S[sb]);
            ++b;
          }
        }
        W.UKEQ[j] = exp(-ds + dh - lP * dnu[j]);
      } else if (kind == 2) {
        const int s = rs[j];
        W.UKEQ[j] = exp(M.D(L.rev_lnA)[s] + M.D(L.rev_beta)[s] * logT - M.D(L.rev_eor)[s] * uT);
      }
    }
    const int* ft = M.I(L.fo_type);
    for (int k = lane; k < L.n_fo; k += 32) {
      W.KINF[k] = exp(M.D(L.fo_lnA)[k] + M.D(L.fo_beta)[k] * logT - M.D(L.fo_eor)[k] * uT);
      const double a = M.D(L.fo_a)[k], b = M.D(L.fo_b)[k], c = M.D(L.fo_c)[k], d = M.D(L.fo_d)[k];
      if (ft[k] == 1) {
        const double v = (d != 0.) ? (1. - a) * exp(-T / b) + a * exp(-T / c) + exp(-d / T)
                                   : (1. - a) * exp(-T / b) + a * exp(-T / c);
        W.LOGF[k] = (v < 1.e-300) ? -300. : log10(v);
      } else if (ft[k] == 2) {
        W.LOGF[k] = a * exp(-b / T) + exp(-T / c);
      } else {
        W.LOGF[k] = 0.;
      }
    }
  }
  if (L.n_plog > 0 || L.n_cheb > 0) {
    // pressure-logarithmic and Chebyshev reactions: k depends on P too, so every call
    // (KineticsMap_CHEMKIN.hpp:1332-1348)
    const double Pk = cv ? cTot * kRgas * T : P0;
    const double logTk = log(T);
    const int* prx = M.I(L.plog_rxn);
    __syncwarp();   // after the Arrhenius values other lanes wrote above
    for (int k = lane; k < L.n_plog; k += 32) W.KARR[prx[k]] = plog_k(M, L, k, T, logTk, Pk);
    const int* crx = M.I(L.cheb_rxn);
    for (int k = lane; k < L.n_cheb; k += 32) W.KARR[crx[k]] = cheb_k(M, L, k, T, Pk);
  }
  const double cTotSum = seq_sum(cl, NC);
  __syncwarp();
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
    for (int j = lane; j < NR; j += 32) {
      double kArr = W.KARR[j];
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
        for (int q2 = tp[tb]; q2 < tp[tb + 1]; ++q2) Mc += W.C[ts[q2]] * te[q2];
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
          for (int q2 = fp[fo]; q2 < fp[fo + 1]; ++q2) Mc += W.C[fs[q2]] * fe[q2];
        } else {
          Mc = W.C[single] + 1.e-16;
        }
        const double kInf = W.KINF[fo];
        const double lF = W.LOGF[fo];
        const double Pr = kArr * Mc / kInf;
        const bool cabr = M.I(L.fo_cabr)[fo] != 0;
        double wF = 1.;
        const int ty = M.I(L.fo_type)[fo];
        if (ty == 1) {
          if (Pr > 1.e-32 || cabr) {
            const double nTroe = 0.75 - 1.27 * lF;
            const double cTroe = -0.4 - 0.67 * lF;
            const double sTroe = log10(Pr) + cTroe;
            const double qq = sTroe / (nTroe - 0.14 * sTroe);
            wF = pow(10., lF / (1. + qq * qq));
          } else {
            const double qq = 1. / 0.14;
            wF = pow(10., lF / (1. + qq * qq));
          }
        } else if (ty == 2) {
          const double l10 = log10(Pr);
          const double xSRI = 1. / (1. + l10 * l10);
          wF = pow(lF, xSRI) * M.D(L.fo_d)[fo];
          const double e = M.D(L.fo_e)[fo];
          if (e != 0.) wF *= pow(T, e);
        }
        // CABR (KineticsMap_CHEMKIN.hpp:1613-1660): k0 (1 / (1 + Pr)) F; fall-off: k_inf (Pr / (1 + Pr)) F
        const double corr = cabr ? (1. / (1. + Pr)) * wF : kInf * (Pr / (1. + Pr)) * wF / kArr;
        kMod *= corr;
      }
      if (L.n_xfo > 0) {     // extended fall-off (KineticsMap_CHEMKIN.hpp:1672-1681)
        const int xs = M.I(L.xfo_slot)[j];
        if (xs >= 0) {
          kArr = xfo_k(M, L, xs, T, cTotSum, [&](int k) { return W.C[k]; });
          kMod = kArr;
        }
      }
      double fwd = 1.;
      for (int q2 = op[j]; q2 < op[j + 1]; ++q2) fwd *= conc_factor(onu[q2], W.C[osp[q2]]);
      double net = fwd;
      const int kind = rk[j];
      if (kind != 0) {
        double rv = 1.;
        for (int q2 = pp[j]; q2 < pp[j + 1]; ++q2) rv *= conc_factor(pnu[q2], W.C[psp[q2]]);
        if (kind == 1) rv *= W.UKEQ[j];
        else rv *= W.UKEQ[j] / kArr;
        net -= rv;
      }
      net *= kMod;
      if constexpr (kDrg) {
        if (W.DROP[j]) net = 0.;   // DRG-reduced system: dropped reactions (chemistry_DRG.H)
      }
      W.NET[j] = net;
    }
  }
  __syncwarp();
  double Rl = 0.;
  if (lane < NC) {
    const int* fp = M.I(L.fr_ptr);
    const int* fr = M.I(L.fr_rxn);
    const double* fc = M.D(L.fr_coef);
    double rate = 0.;
    for (int q2 = fp[lane]; q2 < fp[lane + 1]; ++q2) {
      const double c = fc[q2];
      rate += contrib(c < 0. ? -c : c, W.NET[fr[q2]]) * (c < 0. ? -1. : 1.);
    }
    Rl = rate;
  }
  double dyl = lane < NC ? mwl * Rl / rho : 0.;
  double QR = W.SC[1];
  if (energy) {
    double cpl = 0.;
    if (lane < NC) {
      const double* HT = M.D(L.cp_ht) + 5 * lane;
      const double* LT = M.D(L.cp_lt) + 5 * lane;
      const double* A = T > TM[lane] ? HT : LT;
      cpl = A[0] + T * A[1] + T2 * A[2] + T3 * A[3] + T4 * A[4];
    }
    double cpm = seq_sum(cpl * xl, NC);
    cpm *= kRgas;
    const double d = seq_sum(Rl * hl, NC);
    QR = -d * kRgas * T;
    if (cv) {
      const double CvMixMass = (cpm - kRgas) / MWmix;
      const double sumR = seq_sum(Rl, NC);
      if (lane == NC) dyl = (QR + kRgas * T * sumR) / (rho0 * CvMixMass);
    } else {
      const double CpMixMass = cpm / MWmix;
      if (lane == NC) dyl = QR / (rho * CpMixMass);
    }
  } else if (lane == NC) {
    dyl = 0.;
  }
  __syncwarp();
  if (lane == 0) W.SC[1] = QR;
  __syncwarp();
  return dyl;
}

// ---------------------------------------------------------------------------
// Gear / multivalue BDF integrator state for one warp (one cell).  Vectors are
// held one component per lane (registers) or in the per-warp shared arrays.
// ---------------------------------------------------------------------------
// kDrg: the DRG-reduced system (chemistry_DRG.H) instead of the full reactor.
template <bool kDrg = false>
struct GearWarpT {
  static constexpr int MAX_ORDER = 5, MIN_ORDER = 1;
  enum { H_DEC, H_CONST, H_INC };
  enum { O_DEC, O_CONST, O_INC };
  enum { JAC_CHANGE, JAC_MODIFIED };
  enum { M_TO_FACT, M_FACT };
  enum { CONV_FAIL, CONV_OK };

  const MechLayout* L;
  const double* Md;
  const int* Mi;
  double* ws;
  WarpWS W;
  int lane, ne;
  bool active;        // lane < ne
  // per-lane vector components
  double b, deltab, f, va, vb, y, y0, eps, minv, maxv;
  // scalar state (replicated in all lanes)
  double alfa2_4, alfa2_5;   // alfa2[4], alfa2[5]; alfa2[0..3] stay 0.8
  __device__ __forceinline__ double alfa2(unsigned k) const { return k == 4 ? alfa2_4 : (k == 5 ? alfa2_5 : .8); }
  double abs_tol, rel_tol;
  unsigned maximum_order, max_number_steps;
  double t, t0, tOut, tInMeshPoint, tStabilize;
  double hPreviousStep, hNordsieck, hScaleMax, h, hNextStep, hScale;
  bool fixedOrderMin;
  unsigned iterConstSteps, iterMinimumOrder;
  unsigned p, iterOrder, orderInNextStep, maxConvergenceIterations, maxIterationsJacobian;
  int odeHStatus, odeOrderStatus, status, factorizationStatus, jacobianStatus, convergenceStatus;
  unsigned numberOfSteps, iterConvergence, iterConvergenceRate, iterConvergenceFailure, iterErrorFailure;
  unsigned numberOfConvergenceFailuresForOrderMax, stepOfLastJacobian;
  long long cnt[NCNT];
  // DRG-reduced system (BatchReactorHomogeneousConstantPressure.H:253-320): lane l < drg_ni owns species
  // drg_sp (the l-th important one), lane drg_ni owns T; as a lane of the full layout (species `lane`),
  // drg_pos is that species' reduced index or -1, drg_omega its fixed mass fraction.
  bool unconstrained = false;   // no minimum/maximum constraints: KernelDense's unconstrained increments
  int drg_ni = 0, drg_sp = 0, drg_pos = -1, drg_nc = 0;
  double drg_omega = 0.;

  __device__ __forceinline__ double& Z(int i) { return W.Z[i * 32 + lane]; }
  __device__ __forceinline__ double& V(int i) { return W.V[i * 32 + lane]; }

  // f(y) of the system being integrated: the full reactor, or the DRG-reduced one evaluated through the
  // full layout (kept species fixed, dropped reactions at zero rate) and gathered back to the reduced lanes
  __device__ __forceinline__ double eval(double yl) {
    if constexpr (!kDrg) {
      return rhs_warp<false>(L, Md, Mi, ws, yl, __shfl_sync(kFull, yl, ne - 1));
    } else {
      const double T = __shfl_sync(kFull, yl, drg_ni);
      const double v = __shfl_sync(kFull, yl, drg_pos >= 0 ? drg_pos : 0);
      const double yf = lane < drg_nc ? (drg_pos >= 0 ? v : drg_omega) : T;
      const double df = rhs_warp<true>(L, Md, Mi, ws, yf, T);
      return __shfl_sync(kFull, df, drg_sp);
    }
  }

  __device__ __forceinline__ double rhs(double yl) {
    ++cnt[CNT_RHS];
    return eval(yl);
  }

  __device__ __forceinline__ double error_control(double w, double e) {   // OpenSMOKEUtilities.hpp:689-701
    const double c = active ? w * e : 0.;
    const double s = seq_sum(c * c, ne);
    return sqrt(s / double(ne));
  }

  __device__ __forceinline__ void check_constraints(double& yl) {
    if (active) {
      if (yl < minv) yl = minv;
      if (yl > maxv) yl = maxv;
    }
  }

  __device__ __forceinline__ void one_over_epsilon(double w) {
    if (active) {
      eps = abs_tol + rel_tol * fabs(w);
      eps = 1. / eps;
    }
  }

  // KernelDense::NumericalJacobian, constrained branch (max constraints are on)
  __device__ __forceinline__ void numerical_jacobian(double& yl, double fl) {
    const double ZERO_DER = sqrt(kTinyFloat);
    const double ETA2 = sqrt(kMachEpsDouble);
    const double BETA = 1.e+3 * kMachEpsDouble;
    double hf = BETA * fabs(h) * error_control(fl, eps) * double(ne);
    if (hf < 1.e-10) hf = 1.;
    const int n = ne;
    for (int j = 0; j < n; ++j) {
      const double yh = __shfl_sync(kFull, yl, j);
      const double ej = __shfl_sync(kFull, eps, j);
      const double mxj = __shfl_sync(kFull, maxv, j);
      double hJ;
      if (kDrg && unconstrained) {   // KernelDense.hpp:111-193 without maximum constraints
        hJ = ETA2 * fabs(fmax(yh, 1. / ej));
        const double hJf = hf / ej;
        hJ = fmax(hJ, hJf);
        hJ = fmax(hJ, ZERO_DER);
        hJ = fmin(hJ, 0.001 + 0.001 * fabs(yh));
      } else {
        const double a = fabs(yh), bb = fabs(1. / ej);
        hJ = ETA2 * (a > bb ? a : bb);
        const double hJf = hf / ej;
        hJ = fmax(hJ, hJf);
        hJ = fmax(hJ, ZERO_DER);
        if (yh + hJ > mxj) hJ = -hJ;
      }
      const double saved = yl;
      if (lane == j) yl += hJ;
      const double aux = eval(yl);
      ++cnt[CNT_JAC_RHS];
      yl = saved;
      const double hInv = 1. / hJ;
      if (active) W.J[lane * (n + 1) + j] = hInv * (aux - fl);
    }
    __syncwarp();
  }

  // G = I - hr0 J; partial-pivot LU (largest magnitude, first occurrence)
  __device__ __forceinline__ void build_and_factorize(double hr0) {
    const int n = ne, ld = n + 1;
    if (active) {
      for (int j = 0; j < n; ++j) {
        double g = W.J[lane * ld + j];
        g *= -hr0;
        if (j == lane) g += 1.;
        W.G[lane * ld + j] = g;
      }
    }
    __syncwarp();
    for (int k = 0; k < n; ++k) {
      // pivot search over rows k..n-1 of column k, ties -> lowest row
      double best = (lane >= k && lane < n) ? fabs(W.G[lane * ld + k]) : -1.;
      int row = lane;
      for (int off = 16; off > 0; off >>= 1) {
        const double ob = __shfl_down_sync(kFull, best, off);
        const int orow = __shfl_down_sync(kFull, row, off);
        if (ob > best || (ob == best && orow < row)) { best = ob; row = orow; }
      }
      const int pr = __shfl_sync(kFull, row, 0);
      if (lane == 0) W.PIV[k] = pr;
      __syncwarp();
      if (pr != k) {
        for (int j = lane; j < n; j += 32) {
          const double tmp = W.G[k * ld + j];
          W.G[k * ld + j] = W.G[pr * ld + j];
          W.G[pr * ld + j] = tmp;
        }
      }
      __syncwarp();
      const double d = W.G[k * ld + k];
      if (lane > k && lane < n) {
        double l = W.G[lane * ld + k];
        if (d != 0.) l /= d;
        W.G[lane * ld + k] = l;
        for (int j = k + 1; j < n; ++j) W.G[lane * ld + j] -= l * W.G[k * ld + j];
      }
      __syncwarp();
    }
    ++cnt[CNT_FACT];
  }

  __device__ __forceinline__ void solve(double& xl) {   // KernelDense::SolveLinearSystem
    const int n = ne, ld = n + 1;
    for (int k = 0; k < n; ++k) {
      const int pk = W.PIV[k];
      if (pk != k) {
        const double a = __shfl_sync(kFull, xl, k);
        const double c = __shfl_sync(kFull, xl, pk);
        if (lane == k) xl = c;
        if (lane == pk) xl = a;
      }
    }
    for (int j = 0; j < n; ++j) {
      const double v = __shfl_sync(kFull, xl, j);
      if (lane > j && lane < n) xl -= W.G[lane * ld + j] * v;
    }
    for (int j = n - 1; j >= 0; --j) {
      if (lane == j) xl /= W.G[j * ld + j];
      const double v = __shfl_sync(kFull, xl, j);
      if (lane < j) xl -= W.G[lane * ld + j] * v;
    }
    ++cnt[CNT_SOLVE];
  }

  __device__ __forceinline__ void set_initial_conditions(double tstart, double y0l) {
    tOut = t = t0 = tInMeshPoint = tStabilize = tstart;
    p = 1; iterOrder = 0; orderInNextStep = 1; maxConvergenceIterations = 4;
    maxIterationsJacobian = 20 + 5 * (unsigned)(ne - 3);
    if (maxIterationsJacobian > 50u && ne < 80) maxIterationsJacobian = 50u;
    odeHStatus = H_CONST; odeOrderStatus = O_CONST; status = 1;
    factorizationStatus = M_TO_FACT; jacobianStatus = JAC_CHANGE; convergenceStatus = CONV_OK;
    h = 0.; hNextStep = 0.; hScale = 0.;
    numberOfSteps = 0; numberOfConvergenceFailuresForOrderMax = 0;
    iterConvergence = 0; iterConvergenceRate = 0; iterConvergenceFailure = 0; iterErrorFailure = 0;
    stepOfLastJacobian = 0;
    y0 = y0l;
    hPreviousStep = 0.; hNordsieck = 0.; hScaleMax = 1000.;
    fixedOrderMin = false; iterConstSteps = 0; iterMinimumOrder = 0;
    for (int k = 0; k < NCNT; ++k) cnt[k] = 0;
    f = rhs(y0);
  }

  __device__ __forceinline__ unsigned find_correction() {
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
    const double r0 = c_gear.r[0][p - 1];
    const double hr0 = h * r0;
    if (factorizationStatus == M_FACT && iterOrder == 0) factorizationStatus = M_TO_FACT;
    if (factorizationStatus == M_TO_FACT) {
      build_and_factorize(hr0);
      factorizationStatus = M_FACT;
    }
    deltab = f * h;
    deltab -= active ? V(1) : 0.;
    solve(deltab);
    b = deltab;
    double oldCC = 0.;
    for (unsigned k = 1; k <= maxConvergenceIterations; ++k) {
      const double cc = r0 * error_control(deltab, eps);
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
      solve(deltab);
      b += deltab;
    }
    convergenceStatus = CONV_FAIL;
    return maxConvergenceIterations;
  }

  __device__ __forceinline__ void convergence_failure_recovery() {
    hScale = 0.25;
    if (numberOfSteps < 10) hScale = 0.1;
    hScale = fmax(hScale, 0. / fabs(h));
    odeHStatus = H_DEC;
    if (p > (unsigned)MIN_ORDER) { p -= 1; odeOrderStatus = O_DEC; }
    alfa2_4 -= 0.01;
    alfa2_5 -= 0.02;
    if (alfa2_4 < 0.) { alfa2_4 = 0.; maximum_order = 3; if (p > 3) { p = 3; odeOrderStatus = O_DEC; } }
    if (alfa2_5 < 0.) { alfa2_5 = 0.; maximum_order = 4; if (p > 4) { p = 4; odeOrderStatus = O_DEC; } }
    if (numberOfSteps > 5) {
      numberOfConvergenceFailuresForOrderMax++;
      if (numberOfConvergenceFailuresForOrderMax % 5 == 0) {
        if (p != (unsigned)MIN_ORDER) { p = MIN_ORDER; odeOrderStatus = O_DEC; }
      }
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

  __device__ __forceinline__ void convergence_rate() {
    if (iterErrorFailure > 0 || iterConvergenceFailure > 0) iterConvergenceRate = 0;
    if (iterConvergence <= 1) return;
    const int n = ne, ld = n + 1;
    vb = active ? V(0) - Z(0) : 0.;
    // J * vb, row l accumulated over columns in order
    double s = 0.;
    for (int j = 0; j < n; ++j) {
      const double vj = __shfl_sync(kFull, vb, j);
      if (active) s += W.J[lane * ld + j] * vj;
    }
    va = s;
    va *= h;
    va += active ? Z(1) : 0.;
    va = (active ? V(1) : 0.) - va;
    const double normd = seq_sum(active ? fabs(va) : 0., n);
    const double normf = seq_sum(active ? fabs(V(1)) : 0., n);
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

  __device__ __forceinline__ void multi_value_step() {
    if (active) {
      for (unsigned i = 0; i <= p; ++i) V(i) = Z(i);
      for (int i = 0; i < int(p); ++i)
        for (int j = int(p) - 1; j >= i; --j) V(j) += V(j + 1);
      if (V(0) < minv) {
        if (fabs(V(0) - minv) * eps < double(ne)) {
          V(0) = minv; V(1) = minv - Z(0);
          for (unsigned i = 2; i <= p; ++i) V(i) = 0.;
        }
      }
      if (V(0) > maxv) {
        if (fabs(V(0) - maxv) * eps < double(ne)) {
          V(0) = maxv; V(1) = maxv - Z(0);
          for (unsigned i = 2; i <= p; ++i) V(i) = 0.;
        }
      }
    }
    __syncwarp();
    iterConvergence = find_correction();
    if (convergenceStatus == CONV_FAIL) return;
    const double r0 = c_gear.r[0][p - 1];
    if (active) {
      va = b * r0;
      if (V(0) + va < minv) {
        b = minv - Z(0) - V(1);
        V(0) = minv - va;
        if (V(0) < minv) V(0) = minv;
      }
      if (V(0) + va > maxv) {
        b = maxv - Z(0) - V(1);
        V(0) = maxv - va;
        if (V(0) > maxv) V(0) = maxv;
      }
      V(0) += va;
      V(1) += b;
      for (unsigned i = 2; i <= p; ++i) {
        va = b * c_gear.r[i][p - 1];
        V(i) += va;
      }
      va = V(p) - Z(p);
      V(p + 1) = va / (double(p) + 1.);
      if (iterOrder >= p) {
        va = V(p + 1) - Z(p + 1);
        V(p + 2) = va / (double(p) + 2.);
      }
    }
    __syncwarp();
  }

  __device__ __forceinline__ void new_order_new_h() {
    double hMinus = 0., hCur = 0., hPlus = 0., alfa1 = 0., alfa3 = 0.;
    if (p > (unsigned)MIN_ORDER && odeOrderStatus != O_INC) {
      hMinus = c_gear.Ep[p - 1] * error_control(active ? V(p) : 0., eps) + kMachEpsFloat;
      hMinus = 1. / hMinus;
      alfa1 = alfa2(p - 1) - .05;
      hMinus = alfa1 * pow(hMinus, 1. / double(p));
    }
    {
      hCur = c_gear.Ep[p] * error_control(active ? V(p + 1) : 0., eps) + kMachEpsFloat;
      hCur = 1. / hCur;
      hCur = alfa2(p) * pow(hCur, 1. / double(p + 1));
    }
    if (p < maximum_order && odeOrderStatus != O_DEC) {
      hPlus = c_gear.Ep[p + 1] * error_control(active ? V(p + 2) : 0., eps) + kMachEpsFloat;
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
      if (p > (unsigned)MIN_ORDER) {
        fixedOrderMin = true; iterMinimumOrder = 0;
        orderInNextStep = MIN_ORDER; odeOrderStatus = O_DEC;
        hScale = 0.5; hNextStep = h * hScale; odeHStatus = H_DEC;
      }
    }
  }

  __device__ __forceinline__ void driver_step() {
    iterConvergenceFailure = 0; iterErrorFailure = 0; convergenceStatus = CONV_OK;
    if (odeOrderStatus != O_CONST || odeHStatus != H_CONST) iterOrder = 0;
    p = orderInNextStep;
    odeOrderStatus = O_CONST;
    hScaleMax = 2.;
    if (numberOfSteps < 10) hScaleMax = 1000.;
    else if (numberOfSteps > 10 && numberOfSteps < 20) hScaleMax = 10.;
    for (int guard = 0; guard < 1000000; ++guard) {
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
      __syncwarp();
      multi_value_step();
      if (convergenceStatus == CONV_FAIL) {
        iterConvergenceFailure++;
        ++cnt[CNT_CONVFAIL];
        if (iterConvergenceFailure >= 50u) { status = -5; return; }
        if (fabs(h - 0.) <= kMachEpsDouble * 0.) { status = -6; return; }
        convergence_failure_recovery();
      } else {
        double hCur = c_gear.Ep[p] * error_control(active ? V(p + 1) : 0., eps);
        if (hCur > 1.) {
          iterErrorFailure++;
          ++cnt[CNT_ERRFAIL];
          if (iterErrorFailure >= 50u) { status = -4; return; }
          if (fabs(h - 0.) <= kMachEpsDouble * 0.) { status = -6; return; }
          hScaleMax = 1.;
          hCur = 0.8 * pow(1. / hCur, 1. / double(p + 1));
          hScale = hCur;
          if (p > (unsigned)MIN_ORDER) {
            double hMinus = c_gear.Ep[p - 1] * error_control(active ? V(p) : 0., eps);
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
          hNordsieck = h; hPreviousStep = h; hNextStep = h;
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
          __syncwarp();
          return;
        }
      }
      __syncwarp();
    }
    status = -5;
  }

  // MultiValueSolver::Solve from a fresh initial condition.  On failure y holds
  // the last accepted state.
  __device__ __forceinline__ int solve_to(double tEnd) {
    tOut = tEnd;
    const bool illegal = active && (y0 < minv || y0 > maxv);
    if (__any_sync(kFull, illegal)) { status = -9; y = y0; return status; }
    one_over_epsilon(y0);
    double lo, hi;
    if (t0 != 0.) { lo = 100. * kMachEpsDouble * fabs(t0); hi = fabs(t0); }
    else { lo = kMachEpsDouble; hi = 1.e-4; }
    double h0 = 0.5 / (error_control(f, eps) + kMachEpsFloat);
    if (h0 < lo) h0 = lo;
    if (h0 > hi) h0 = hi;
    h0 *= fabs(tOut - t0) / (tOut - t0);
    if (active) { Z(0) = y0; Z(1) = f * h0; }
    hPreviousStep = h0; hNordsieck = h0; hNextStep = h0;
    status = 2;
    __syncwarp();
    for (unsigned k = 1; k <= max_number_steps; ++k) {
      one_over_epsilon(active ? Z(0) : 0.);
      const double tolSafe = kMachEpsDouble * error_control(active ? Z(0) : 0., eps);
      if (tolSafe > 1.) { status = -2; y = active ? Z(0) : 0.; return status; }
      tInMeshPoint = t;
      driver_step();
      if (status <= 0) { t = tInMeshPoint; y = active ? Z(0) : 0.; return status; }
      numberOfSteps++;
      ++cnt[CNT_STEPS];
      if (tOut == t) { y = active ? Z(0) : 0.; return status; }
      if (tOut < t) {
        // Interpolation (:687-706) + the extra RHS call that sets QR at tOut
        const double hp = (tOut - t) / hNordsieck;
        double hr = 1.;
        y = active ? Z(0) : 0.;
        if (hp != 0.) {
          for (unsigned i = 1; i <= p; ++i) {
            hr *= hp;
            if (active) { va = Z(i) * hr; y += va; }
          }
          check_constraints(y);
        }
        va = rhs(y);
        return status;
      }
    }
    status = -1;
    y = active ? Z(0) : 0.;
    return status;
  }
};
using GearWarp = GearWarpT<false>;

}  // namespace lsg
