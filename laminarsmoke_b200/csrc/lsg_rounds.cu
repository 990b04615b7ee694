// Batched reaction step, round scheme.  Every cell of the batch keeps its
// whole solver state in one contiguous record in HBM, and the step advances in
// rounds, each a fixed sequence of kernels over the list of cells that are
// still integrating:
//
//   rhs       one thread per cell evaluates the RHS the cell asked for (f(y0),
//             the predictor, a Newton iterate, a stabilisation call or the
//             final call at tOut), or all n perturbed RHS of a
//             finite-difference Jacobian and the Jacobian itself: the
//             reaction loop runs convergent across the warp, with the
//             mechanism tables staged once per block into shared memory by a
//             bulk copy;
//   advance   one warp per cell (lane = ODE component) consumes the result and
//             runs the cell's Gear/BDF solver to its next RHS request or to
//             the end of its integration: the record is loaded in one coalesced
//             pass, every vector operation is lane-parallel, norms are warp
//             tree reductions; a factorisation of G = I - h r0 J (partial
//             pivoting, FP32 or FP64) is done by the warp in shared memory and
//             turned into G^-1 (one column per lane), so every Newton solve is
//             one matrix-vector product whose broadcasts are independent;
//   compact   the cells still integrating form the next round's list
//             (order-preserving inside each warp).
//
// The method is the one of the plain step -- MultiValueSolver.hpp:423-1328,
// MethodGear.hpp:195-516, KernelDense.hpp:111-245 (under
// solvers/openSMOKEpp4laminarSMOKE/math/native-ode-solvers) -- with the RHS of
// BatchReactorHomogeneousConstantPressure.H:175-223.  The Jacobian is stored in
// FP64 whatever the precision of the factors.  With FP32 factors every linear
// solve is refined against its FP64 residual (G = I - h r0 J applied in FP64
// from the stored FP64 Jacobian).
#include "lsg_common.cuh"
#include "lsg_kernels.h"

namespace lsg {

static __constant__ GearConsts c_gear_r;

namespace {

constexpr int kRT = 128;       // threads per block of the RHS kernel (one cell each)
constexpr int kWA = 4;         // warps per block of the advance kernel (one cell each)
constexpr int kAT = 128;       // threads per block of the init kernel
constexpr int kCT = 256;       // threads per block of the compaction kernel
constexpr int kRefineR = 1;    // refinement sweeps of a solve with FP32 factors
constexpr int kBins = 6;       // solver-path bins of the compaction
// Row stride (elements) of the per-group matrices in shared memory (G^-1, J): odd, so the lanes of a group
// reading one column (lane = row) hit distinct banks; at most n + 1, the stride the buffers are sized for.
__host__ __device__ constexpr int row_ld(int n) { return n | 1; }

enum Phase : int {
  PH_DONE = 0,
  PH_INIT,       // f(y0)
  PH_PRED,       // f(vb), first Newton evaluation
  PH_JAC,        // f(vb + hJ_j e_j) for every column j: the whole FD Jacobian in one visit
  PH_NEWTON,     // f(va), Newton iterate
  PH_STAB_CONV,  // f(z0) during convergence-failure recovery
  PH_STAB_ERR,   // f(z0) after an error-test failure
  PH_FINAL,      // f(y(tOut)) -> QR
};

__device__ __forceinline__ bool rhs_phase(int ph) { return ph >= PH_INIT && ph <= PH_FINAL; }

// scalar state of a cell: doubles D_* at the record start, ints I_* after them
enum : int {
  D_T = 0, D_T0, D_TOUT, D_TMESH, D_TSTAB, D_H, D_HNEXT, D_HNORD, D_HSCALE, D_HSCALEMAX,
  D_A24, D_A25, D_QR, D_OLDCC, D_HF, D_HJ, D_PENDHS, D_HR0, ND_
};
enum : int {
  I_PHASE = 0, I_STATUS, I_P, I_ITORDER, I_ORDNEXT, I_MAXITJ, I_HSTAT, I_OSTAT, I_FACTORIZED, I_JACCHANGE,
  I_CONVOK, I_NSTEPS, I_ITCONV, I_ITCONVRATE, I_ITCONVFAIL, I_ITERRFAIL, I_NCFOM, I_STEPLASTJ, I_ITCONST,
  I_ITMINORD, I_FIXEDMIN, I_NEWTONK, I_JCOL, I_MAXORD, I_CNT0, NI_ = I_CNT0 + NCNT
};

// Record of one cell (offsets in doubles from the record start; RS doubles per
// record, a multiple of 32 so records start on 256-byte boundaries):
//   [0, ND_)            scalar doubles
//   [ND_, ND_ + NI_/2)  scalar ints
//   oz   z[8][n]  Nordsieck array      ov   v[8][n]
//   ob, of, of0, ova, ovb, oeps         n each
//   ojac J[n][n] double (row major)     oinv G^-1[n][n] LUT (row major)
struct RecLayout {
  int oz, ov, ob, of, of0, ova, ovb, oeps, ojac, oinv, RS;
};

__host__ __device__ inline RecLayout rec_layout(int n, bool lu64) {
  RecLayout r{};
  int o = ND_ + NI_ / 2;
  r.oz = o; o += 8 * n;
  r.ov = o; o += 8 * n;
  r.ob = o; o += n;
  r.of = o; o += n;
  r.of0 = o; o += n;
  r.ova = o; o += n;
  r.ovb = o; o += n;
  r.oeps = o; o += n;
  r.ojac = o; o += n * n;
  r.oinv = o; o += lu64 ? n * n : (n * n + 1) / 2;
  r.RS = (o + 31) & ~31;
  return r;
}

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


// ---------------------------------------------------------------------------
// Thread-serial RHS of the constant-pressure reactor
// (BatchReactorHomogeneousConstantPressure.H:175-223).  y: this cell's input
// vector (stride ns) with component pj replaced by pval when pj >= 0; f: output.
// C (concentrations), G (h/RT - s/R) and R (formation rates) scratch in shared
// memory, [species][thread].  f has stride fs.  Returns QR.  rho0 > 0 selects
// the constant-volume reactor of that density (BatchReactorHomogeneousConstant
// Volume.H:148-199): cTot = rho0 / MW, dY/dt = MW R / rho0 and
// dT/dt = (QR + R T sum R_i) / (rho0 cv).  With kSources, f receives the
// source terms R_i MW_i instead of the species derivatives (the steady
// solvers' reactionSourceTerms).
// ---------------------------------------------------------------------------
template <bool kSources = false>
__device__ __noinline__ double rhs_cell(const MechLayout* __restrict__ Lp, const double* __restrict__ Md,
                                        const int* __restrict__ Mi, double* __restrict__ scratch,
                                        const double* __restrict__ y, long ns, int pj, double pval,
                                        double* __restrict__ f, long fs, double P0, int energy, double rho0) {
  const MechLayout& L = *Lp;
  const MechView M{Md, Mi};
  const int NC = L.nc, NR = L.nr;
  const int tid = threadIdx.x;
  double* C = scratch;
  double* G = scratch + NC * kRT;        // h/RT - s/R of each species
  double* R = scratch + 2 * NC * kRT;
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
  const bool cv = rho0 > 0.;
  const double cTot = cv ? rho0 / MWmix : P0 / kRgas / T;
  const double rho = cv ? rho0 : cTot * MWmix;
  const double Pk = cv ? cTot * kRgas * T : P0;   // the kinetics map's pressure (PLOG)
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
    const double hrt = A[0] + T * A[1] + T2 * A[2] + T3 * A[3] + T4 * A[4] + uT * A[5];
    const double* B = hi ? M.D(L.ds_ht) + 6 * i : M.D(L.ds_lt) + 6 * i;
    SC_(G, i) = hrt - (B[0] * logT + T * B[1] + T2 * B[2] + T3 * B[3] + T4 * B[4] + B[5]);
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
  const int* op = M.I(L.ford_ptr);     // forward rate-law orders (FORD, else the coefficients)
  const int* osp = M.I(L.ford_sp);
  const double* onu = M.D(L.ford_val);
  const int* pp = M.I(L.prod_ptr);
  const int* psp = M.I(L.prod_sp);
  const double* pnu = M.D(L.prod_nu);
  for (int j = 0; j < NR; ++j) {
    double kArr = exp(lnA[j] + beta[j] * logT - eor[j] * uT);
    if (sgn[j] < 0) kArr *= -1.;
    if (L.n_plog > 0) {   // pressure-logarithmic reaction (KineticsMap_CHEMKIN.hpp:1341-1348)
      const int ps = M.I(L.plog_slot)[j];
      if (ps >= 0) kArr = plog_k(M, L, ps, T, logT, Pk);
    }
    if (L.n_cheb > 0) {   // Chebyshev reaction (KineticsMap_CHEMKIN.hpp:1332-1339)
      const int cs = M.I(L.cheb_slot)[j];
      if (cs >= 0) kArr = cheb_k(M, L, cs, T, Pk);
    }
    if (L.n_xplog > 0) {  // extended PLOG (KineticsMap_CHEMKIN.hpp:1662-1670)
      const int xs = M.I(L.xplog_slot)[j];
      if (xs >= 0) kArr = xplog_k(M, L, xs, T, logT, Pk, cTotSum, [&](int k) { return SC_(C, k); });
    }
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
      const bool cabr = M.I(L.fo_cabr)[fo] != 0;
      double wF = 1.;
      if (ty == 1) {
        double v = (1. - a) * exp(-T / b) + a * exp(-T / c);
        if (d != 0.) v += exp(-d / T);
        const double lF = (v < 1.e-300) ? -300. : log10(v);
        double qq;
        if (Pr > 1.e-32 || cabr) {
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
      // CABR (KineticsMap_CHEMKIN.hpp:1613-1660): k0 (1 / (1 + Pr)) F; fall-off: k_inf (Pr / (1 + Pr)) F
      if (cabr) kMod *= (1. / (1. + Pr)) * wF;
      else kMod *= kInf * (Pr / (1. + Pr)) * wF / kArr;
    }
    if (L.n_xfo > 0) {    // extended fall-off (KineticsMap_CHEMKIN.hpp:1672-1681)
      const int xs = M.I(L.xfo_slot)[j];
      if (xs >= 0) {
        kArr = xfo_k(M, L, xs, T, cTotSum, [&](int k) { return SC_(C, k); });
        kMod = kArr;
      }
    }
    double fwd = 1.;
    for (int q = op[j]; q < op[j + 1]; ++q) fwd *= conc_factor_r(onu[q], SC_(C, osp[q]));
    double net = fwd;
    const int kind = rk[j];
    if (kind != 0) {
      double rv = 1.;
      for (int q = pp[j]; q < pp[j + 1]; ++q) rv *= conc_factor_r(pnu[q], SC_(C, psp[q]));
      double rf;
      if (kind == 1) {
        // 1/Keq = exp(sum_products nu g - sum_reactants nu g - dnu ln(Patm/RT)), g = h/RT - s/R
        // (StoichiometricMap.hpp:916-1001, KineticsMap_CHEMKIN.hpp:1217-1222, summed per side)
        double dg = 0.;
        for (int q = pp[j]; q < pp[j + 1]; ++q) dg += contrib_r(pnu[q], SC_(G, psp[q]));
        for (int q = rp[j]; q < rp[j + 1]; ++q) dg -= contrib_r(rnu[q], SC_(G, rsp[q]));
        rf = exp(dg - lP * dnu[j]);
      } else {
        const int s = rs[j];
        rf = exp(M.D(L.rev_lnA)[s] + M.D(L.rev_beta)[s] * logT - M.D(L.rev_eor)[s] * uT) / kArr;
      }
      rv *= rf;
      net -= rv;
    }
    net *= kMod;
    for (int q = rp[j]; q < rp[j + 1]; ++q) SC_(R, rsp[q]) -= contrib_r(rnu[q], net);
    for (int q = pp[j]; q < pp[j + 1]; ++q) SC_(R, psp[q]) += contrib_r(pnu[q], net);
  }
  double QR = 0., cpm = 0., dsum = 0.;
  for (int i = 0; i < NC; ++i) {
    const double Ri = SC_(R, i);
    f[(long)i * fs] = kSources ? Ri * MW[i] : MW[i] * Ri / rho;
    if (energy) {
      const bool hi = T > TM[i];
      const double* A = hi ? M.D(L.cp_ht) + 5 * i : M.D(L.cp_lt) + 5 * i;
      const double cpi = A[0] + T * A[1] + T2 * A[2] + T3 * A[3] + T4 * A[4];
      cpm += cpi * (SC_(C, i) / cTot);
      const double* Hc = hi ? M.D(L.dh_ht) + 6 * i : M.D(L.dh_lt) + 6 * i;
      dsum += Ri * (Hc[0] + T * Hc[1] + T2 * Hc[2] + T3 * Hc[3] + T4 * Hc[4] + uT * Hc[5]);
    }
  }
  double dT = 0.;
  if (energy) {
    cpm *= kRgas;
    QR = -dsum * kRgas * T;
    if (cv) {
      const double CvMixMass = (cpm - kRgas) / MWmix;
      double sumR = 0.;
      for (int i = 0; i < NC; ++i) sumR += SC_(R, i);
      dT = (QR + kRgas * T * sumR) / (rho0 * CvMixMass);
    } else {
      const double CpMixMass = cpm / MWmix;
      dT = QR / (rho * CpMixMass);
    }
  }
  f[(long)NC * fs] = dT;
#undef SC_
  return QR;
}


// d/dc of conc_factor_r(nu, c): the derivative of one factor of a product of concentrations
__device__ __forceinline__ double dconc_factor_r(double nu, double c1) {
  if (nu == 1.) return 1.;
  if (nu == 2.) return c1 + c1;
  if (nu == 3.) return 3. * c1 * c1;
  if (nu == 0.5) return c1 > 0. ? 0.5 / sqrt(c1) : 0.;
  return c1 > 0. ? nu * pow(c1, nu - 1.) : 0.;
}

// ---------------------------------------------------------------------------
// Analytic Jacobian, species columns, of the constant-pressure reactor
// (BatchReactorHomogeneousConstantPressure.H:175-223) at the state y (stride
// ns), thread-serial.  The reference builds every column by forward
// differences (KernelDense.hpp:111-193); here the NC species columns are
// exact derivatives and the temperature column stays a forward difference
// (its own work item, jacobian_column).  With c_k = cTot x_k(Y) at fixed T
// (cTot = P/(R T)), x the mole fractions and D = dOmega/dc (Omega the
// formation rates, KineticsMap_CHEMKIN.hpp:1683-1768):
//   dc_k/dY_j = rho (delta_kj - x_k) / MW_j,
//   J_ij = (MW_i / MW_j) (D_ij - sum_k D_ik x_k + Omega_i / cTot)       (i < NC),
//   J_Tj = -(R T MWmix / (MW_j cpm)) sum_k (h/RT)_k (D_kj - s_k)
//          - f_T MWmix (R cp_j - cpm) / (MW_j cpm)                     (energy on),
// s_k = sum_m D_km x_m, cpm the mixture molar cp, f_T = QR / (cTot cpm).
// D collects, per reaction r with net rate q_r = kMod_r (fwd_r - rev_r):
// the partials of the products of concentrations (forward orders, reverse
// coefficients times 1/Keq or k_rev/k_fwd), and through the third-body
// concentration M = sum c + sum (eps - 1) c the partials of kMod (third body:
// kArr; fall-off: kMod [1/(1+Pr) + Pr dlnF/dPr] / M, CABR: kMod [-Pr/(1+Pr) +
// Pr dlnF/dPr] / M, with the Troe and SRI forms' dlnF/dPr).  The part of
// dM/dc_k that is the same for every k (the sum of all concentrations) adds a
// term independent of k to a row of D, which the x-weighted sum removes
// exactly (sum x = 1): only the (eps - 1) terms and single-bath partials are
// accumulated.  J is written row-major into Jg[i * n + j] for j < NC.
// Scratch as rhs_cell: C (concentrations), G (h/RT - s/R, later reused),
// R (formation rates), [species][thread] in shared memory.
// ---------------------------------------------------------------------------
__device__ __noinline__ void analytic_jacobian_species(const MechLayout* __restrict__ Lp, const double* __restrict__ Md,
                                                       const int* __restrict__ Mi, double* __restrict__ scratch,
                                                       const double* __restrict__ y, long ns, double P0, int energy,
                                                       double* __restrict__ Jg) {
  const MechLayout& L = *Lp;
  const MechView M{Md, Mi};
  const int NC = L.nc, NR = L.nr, n = NC + 1;
  const int tid = threadIdx.x;
  double* C = scratch;
  double* G = scratch + NC * kRT;
  double* R = scratch + 2 * NC * kRT;
#define SC_(arr, i) arr[(i) * kRT + tid]
  const double* MW = M.D(L.mw);
  const double T = y[(long)NC * ns];
  double u = 0.;
  for (int i = 0; i < NC; ++i) {
    const double yi = y[(long)i * ns];
    SC_(C, i) = yi;
    u += yi / MW[i];
  }
  const double MWmix = 1. / u;
  const double cTot = P0 / kRgas / T;
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
    const double hrt = A[0] + T * A[1] + T2 * A[2] + T3 * A[3] + T4 * A[4] + uT * A[5];
    const double* B = hi ? M.D(L.ds_ht) + 6 * i : M.D(L.ds_lt) + 6 * i;
    SC_(G, i) = hrt - (B[0] * logT + T * B[1] + T2 * B[2] + T3 * B[3] + T4 * B[4] + B[5]);
    SC_(R, i) = 0.;
  }
  for (int i = 0; i < NC; ++i)
    for (int j = 0; j < NC; ++j) Jg[i * n + j] = 0.;
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
  const int* op = M.I(L.ford_ptr);
  const int* osp = M.I(L.ford_sp);
  const double* onu = M.D(L.ford_val);
  const int* pp = M.I(L.prod_ptr);
  const int* psp = M.I(L.prod_sp);
  const double* pnu = M.D(L.prod_nu);
  // D[i][k] += nu_ij g for every species i of reaction j (reactants negative)
  auto scatter = [&](int j, int k, double g) {
    for (int q = rp[j]; q < rp[j + 1]; ++q) Jg[rsp[q] * n + k] -= contrib_r(rnu[q], g);
    for (int q = pp[j]; q < pp[j + 1]; ++q) Jg[psp[q] * n + k] += contrib_r(pnu[q], g);
  };
  for (int j = 0; j < NR; ++j) {
    double kArr = exp(lnA[j] + beta[j] * logT - eor[j] * uT);
    if (sgn[j] < 0) kArr *= -1.;
    if (L.n_plog > 0) {
      const int ps = M.I(L.plog_slot)[j];
      if (ps >= 0) kArr = plog_k(M, L, ps, T, logT, P0);
    }
    if (L.n_cheb > 0) {
      const int cs = M.I(L.cheb_slot)[j];
      if (cs >= 0) kArr = cheb_k(M, L, cs, T, P0);
    }
    if (L.n_xplog > 0) {
      const int xs = M.I(L.xplog_slot)[j];
      if (xs >= 0) kArr = xplog_k(M, L, xs, T, logT, P0, cTotSum, [&](int k) { return SC_(C, k); });
    }
    double kMod = kArr;
    double dkdM = 0.;          // d kMod / d M
    int mkind = 0;             // 0: no M; 1: third body (efficiency list tb); 2: fall-off mixture; 3: fall-off single bath
    int mslot = -1;
    const int tb = tbs[j];
    if (tb >= 0) {
      double Mc = cTotSum;
      const int* tp = M.I(L.tb_ptr);
      const int* ts = M.I(L.tb_sp);
      const double* te = M.D(L.tb_eff);
      for (int q = tp[tb]; q < tp[tb + 1]; ++q) Mc += SC_(C, ts[q]) * te[q];
      kMod *= Mc;
      dkdM = kArr;
      mkind = 1;
      mslot = tb;
    }
    const int fo = fos[j];
    if (fo >= 0) {
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
        mkind = 2;
      } else {
        Mc = SC_(C, single) + 1.e-16;
        mkind = 3;
      }
      mslot = fo;
      const double Pr = kArr * Mc / kInf;
      const bool cabr = M.I(L.fo_cabr)[fo] != 0;
      double wF = 1., PrdlnF = 0.;   // F and Pr dlnF/dPr
      if (ty == 1) {
        double v = (1. - a) * exp(-T / b) + a * exp(-T / c);
        if (d != 0.) v += exp(-d / T);
        const double lF = (v < 1.e-300) ? -300. : log10(v);
        double qq;
        if (Pr > 1.e-32 || cabr) {
          const double nTroe = 0.75 - 1.27 * lF;
          const double cTroe = -0.4 - 0.67 * lF;
          const double sTroe = log10(Pr) + cTroe;
          const double den = nTroe - 0.14 * sTroe;
          qq = sTroe / den;
          // log10 F = lF / (1 + q^2), dq/ds = n / den^2, Pr dlnF/dPr = d log10 F / d log10 Pr
          const double opq = 1. + qq * qq;
          PrdlnF = -lF * 2. * qq / (opq * opq) * nTroe / (den * den);
        } else {
          qq = 1. / 0.14;
        }
        wF = exp10(lF / (1. + qq * qq));
      } else if (ty == 2) {
        const double lF = a * exp(-b / T) + exp(-T / c);
        const double l10 = log10(Pr);
        const double opl = 1. + l10 * l10;
        const double xSRI = 1. / opl;
        wF = pow(lF, xSRI) * d;
        const double e = M.D(L.fo_e)[fo];
        if (e != 0.) wF *= pow(T, e);
        // ln F = X ln(lF) + ...: Pr dlnF/dPr = ln(lF) dX/dlog10Pr / ln 10
        if (Pr > 1.e-300 && lF > 0.) PrdlnF = log(lF) * (-2. * l10 / (opl * opl)) / 2.302585092994046;
      }
      if (cabr) {
        kMod *= (1. / (1. + Pr)) * wF;
        dkdM = Mc > 0. ? kMod * (-Pr / (1. + Pr) + PrdlnF) / Mc : 0.;
      } else {
        kMod *= kInf * (Pr / (1. + Pr)) * wF / kArr;
        dkdM = Mc > 0. ? kMod * (1. / (1. + Pr) + PrdlnF) / Mc : 0.;
      }
    }
    // forward product and its partials (orders lambda: FORD or the coefficients)
    if (L.n_xfo > 0) {    // extended fall-off (KineticsMap_CHEMKIN.hpp:1672-1681)
      const int xs = M.I(L.xfo_slot)[j];
      if (xs >= 0) {
        kArr = xfo_k(M, L, xs, T, cTotSum, [&](int k) { return SC_(C, k); });
        kMod = kArr;
      }
    }
    double fwd = 1.;
    for (int q = op[j]; q < op[j + 1]; ++q) fwd *= conc_factor_r(onu[q], SC_(C, osp[q]));
    for (int q = op[j]; q < op[j + 1]; ++q) {
      double dp = dconc_factor_r(onu[q], SC_(C, osp[q]));
      for (int q2 = op[j]; q2 < op[j + 1]; ++q2)
        if (q2 != q) dp *= conc_factor_r(onu[q2], SC_(C, osp[q2]));
      scatter(j, osp[q], kMod * dp);
    }
    double net = fwd;
    const int kind = rk[j];
    if (kind != 0) {
      double rv = 1.;
      for (int q = pp[j]; q < pp[j + 1]; ++q) rv *= conc_factor_r(pnu[q], SC_(C, psp[q]));
      double rf;
      if (kind == 1) {
        double dg = 0.;
        for (int q = pp[j]; q < pp[j + 1]; ++q) dg += contrib_r(pnu[q], SC_(G, psp[q]));
        for (int q = rp[j]; q < rp[j + 1]; ++q) dg -= contrib_r(rnu[q], SC_(G, rsp[q]));
        rf = exp(dg - lP * dnu[j]);
      } else {
        const int sr = rs[j];
        rf = exp(M.D(L.rev_lnA)[sr] + M.D(L.rev_beta)[sr] * logT - M.D(L.rev_eor)[sr] * uT) / kArr;
      }
      for (int q = pp[j]; q < pp[j + 1]; ++q) {
        double dp = dconc_factor_r(pnu[q], SC_(C, psp[q]));
        for (int q2 = pp[j]; q2 < pp[j + 1]; ++q2)
          if (q2 != q) dp *= conc_factor_r(pnu[q2], SC_(C, psp[q2]));
        scatter(j, psp[q], -kMod * rf * dp);
      }
      rv *= rf;
      net -= rv;
    }
    // through M: the (eps - 1) efficiencies, or the single bath species
    if (mkind != 0 && dkdM != 0.) {
      const double gm = net * dkdM;
      if (mkind == 1) {
        const int* tp = M.I(L.tb_ptr);
        const int* ts = M.I(L.tb_sp);
        const double* te = M.D(L.tb_eff);
        for (int q = tp[mslot]; q < tp[mslot + 1]; ++q) scatter(j, ts[q], gm * te[q]);
      } else if (mkind == 2) {
        const int* fp = M.I(L.fo_ptr);
        const int* fs = M.I(L.fo_sp);
        const double* fe = M.D(L.fo_eff);
        for (int q = fp[mslot]; q < fp[mslot + 1]; ++q) scatter(j, fs[q], gm * fe[q]);
      } else {
        scatter(j, M.I(L.fo_single)[mslot], gm);
      }
    }
    net *= kMod;
    for (int q = rp[j]; q < rp[j + 1]; ++q) SC_(R, rsp[q]) -= contrib_r(rnu[q], net);
    for (int q = pp[j]; q < pp[j + 1]; ++q) SC_(R, psp[q]) += contrib_r(pnu[q], net);
  }
  // mixture cp and QR (the RHS's), for the temperature row
  double cpm = 0., dsum = 0.;
  if (energy) {
    for (int i = 0; i < NC; ++i) {
      const bool hi = T > TM[i];
      const double* A = hi ? M.D(L.cp_ht) + 5 * i : M.D(L.cp_lt) + 5 * i;
      cpm += (A[0] + T * A[1] + T2 * A[2] + T3 * A[3] + T4 * A[4]) * (SC_(C, i) / cTot);
      const double* Hc = hi ? M.D(L.dh_ht) + 6 * i : M.D(L.dh_lt) + 6 * i;
      dsum += SC_(R, i) * (Hc[0] + T * Hc[1] + T2 * Hc[2] + T3 * Hc[3] + T4 * Hc[4] + uT * Hc[5]);
    }
    cpm *= kRgas;
  }
  const double QR = -dsum * kRgas * T;
  const double fT = energy ? QR / (cTot * cpm) : 0.;
  // rows: s_k, the species rows in place, and t_j = sum_k (h/RT)_k D_kj for the temperature row (in G)
  for (int j = 0; j < NC; ++j) SC_(G, j) = 0.;
  double shs = 0.;
  for (int k = 0; k < NC; ++k) {
    double sk = 0.;
    for (int m = 0; m < NC; ++m) sk += Jg[k * n + m] * (SC_(C, m) / cTot);
    double hk = 0.;
    if (energy) {
      const double* Hc = T > TM[k] ? M.D(L.dh_ht) + 6 * k : M.D(L.dh_lt) + 6 * k;
      hk = Hc[0] + T * Hc[1] + T2 * Hc[2] + T3 * Hc[3] + T4 * Hc[4] + uT * Hc[5];
      shs += hk * sk;
    }
    const double add = SC_(R, k) / cTot - sk;
    for (int m = 0; m < NC; ++m) {
      const double dkm = Jg[k * n + m];
      if (energy) SC_(G, m) += hk * dkm;
      Jg[k * n + m] = (MW[k] / MW[m]) * (dkm + add);
    }
  }
  for (int m = 0; m < NC; ++m) {
    double jt = 0.;
    if (energy) {
      const double* A = T > TM[m] ? M.D(L.cp_ht) + 5 * m : M.D(L.cp_lt) + 5 * m;
      const double cpj = kRgas * (A[0] + T * A[1] + T2 * A[2] + T3 * A[3] + T4 * A[4]);
      jt = -(kRgas * T * MWmix / (MW[m] * cpm)) * (SC_(G, m) - shs) - fT * MWmix * (cpj - cpm) / (MW[m] * cpm);
    }
    Jg[NC * n + m] = jt;
  }
#undef SC_
}

// Asynchronous global -> shared copies (no register staging); completed by cp_async_wait_all.
__device__ __forceinline__ void cp_async4(void* sdst, const void* gsrc) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(sdst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async8(void* sdst, const void* gsrc) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(sdst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
template <typename T>
__device__ __forceinline__ void cp_async_el(T* sdst, const T* gsrc) {
  if (sizeof(T) == 8) cp_async8(sdst, gsrc);
  else cp_async4(sdst, gsrc);
}

// One out-of-line copy of pow for the step-size selection (keeps the solver
// kernel's instruction footprint small).
__device__ __noinline__ double pow_ol(double x, double y) { return pow(x, y); }

// G^-1 for G = I - hr0 J by Gauss-Jordan elimination on [G | I] with partial
// pivoting on the largest magnitude, first occurrence -- the pivots of the
// partial-pivot LU of KernelDense::BuildAndFactorizeMatrixG.  Lane i of the
// group owns row i; each step's updates are independent and loaded in chunks of
// 4.  Js: J rows (shared), As/Ks: work arrays, Xs: G^-1 (shared), Ig: G^-1 in
// the cell record.  Out of line: one copy serves every call site.
template <typename LUT, int W>
__device__ __noinline__ void gj_inverse(const double* Js, LUT* As, LUT* Ks, LUT* Xs, LUT* Ig, double hr0, int n,
                                        int lane, unsigned gm) {
  const int ld = row_ld(n), la = 2 * n + 1, m2 = 2 * n;
  const bool al = lane < n;
  if (al) {
    for (int j = 0; j < n; ++j) {
      double g = -hr0 * Js[lane * ld + j];
      if (j == lane) g += 1.;
      As[lane * la + j] = (LUT)g;
      As[lane * la + n + j] = (j == lane) ? (LUT)1 : (LUT)0;
    }
  }
  __syncwarp(gm);
  for (int k = 0; k < n; ++k) {
    LUT vv = (lane >= k && lane < n) ? (LUT)fabs((double)As[lane * la + k]) : (LUT)-1;
    int r = lane;
    for (int off = W / 2; off > 0; off >>= 1) {
      const LUT ov = __shfl_xor_sync(gm, vv, off, W);
      const int orr = __shfl_xor_sync(gm, r, off, W);
      if (ov > vv || (ov == vv && orr < r)) { vv = ov; r = orr; }
    }
    r = __shfl_sync(gm, r, 0, W);
    if (r < k || r >= n) r = k;   // a NaN column cannot send the pivot outside rows k..n-1
    // swap rows k and r and scale the pivot row into K (lanes = columns)
    const LUT pv = As[r * la + k];
    const LUT ipv = (pv != (LUT)0) ? (LUT)1 / pv : (LUT)0;
    for (int j = lane; j < m2; j += W) {
      const LUT ak = As[k * la + j], ar = As[r * la + j];
      Ks[j] = ar * ipv;
      if (r != k) As[r * la + j] = ak;
    }
    __syncwarp(gm);
    // eliminate column k from every other row (lane = row)
    if (al && lane != k) {
      const LUT fct = As[lane * la + k];
      LUT* Ai = As + lane * la;
      int j = k;
      for (; j + 4 <= m2; j += 4) {
        const LUT a0 = Ai[j], a1 = Ai[j + 1], a2 = Ai[j + 2], a3 = Ai[j + 3];
        const LUT k0 = Ks[j], k1 = Ks[j + 1], k2 = Ks[j + 2], k3 = Ks[j + 3];
        Ai[j] = a0 - fct * k0;
        Ai[j + 1] = a1 - fct * k1;
        Ai[j + 2] = a2 - fct * k2;
        Ai[j + 3] = a3 - fct * k3;
      }
      for (; j < m2; ++j) Ai[j] = Ai[j] - fct * Ks[j];
    }
    __syncwarp(gm);
    for (int j = lane; j < m2; j += W) As[k * la + j] = Ks[j];
    __syncwarp(gm);
  }
  if (al)
    for (int j = 0; j < n; ++j) {
      const LUT g = As[lane * la + n + j];
      Xs[lane * ld + j] = g;
      if (Ig) Ig[lane * n + j] = g;
    }
  __syncwarp(gm);
}

// Tree sum over a lane group of W lanes (mask gm); every lane receives the total.
template <int W>
__device__ __forceinline__ double wsum_g(unsigned gm, double v) {
#pragma unroll
  for (int off = W / 2; off > 0; off >>= 1) v += __shfl_xor_sync(gm, v, off, W);
  return v;
}

// Weighted RMS norm over the group (OpenSMOKEUtilities.hpp:689-701, tree-ordered sum); out of line.
template <int W>
__device__ __noinline__ double wrms_ol(double x, double e, bool al, int n, unsigned gm) {
  const double c = al ? x * e : 0.;
  return sqrt(wsum_g<W>(gm, c * c) / double(n));
}

// sum_j M[lane][j] * y_j (M row-major in shared memory, leading dimension ld); the broadcasts do not
// depend on each other.  Out of line.
template <typename T, int W>
__device__ __noinline__ double rowdot_ol(const T* M, double y, int n, int ld, int lane, unsigned gm) {
  const bool al = lane < n;
  double s0 = 0., s1 = 0.;
  for (int j = 0; j + 1 < n; j += 2) {
    const double y0 = __shfl_sync(gm, y, j, W);
    const double y1 = __shfl_sync(gm, y, j + 1, W);
    if (al) {
      s0 += (double)M[lane * ld + j] * y0;
      s1 += (double)M[lane * ld + j + 1] * y1;
    }
  }
  if (n & 1) {
    const double y0 = __shfl_sync(gm, y, n - 1, W);
    if (al) s0 += (double)M[lane * ld + n - 1] * y0;
  }
  return s0 + s1;
}

// a[i] for a runtime index 0 <= i < 8 without local-memory indexing
__device__ __forceinline__ double get8(const double (&a)[8], unsigned i) {
  double r = a[0];
#pragma unroll
  for (unsigned k = 1; k < 8; ++k)
    if (i == k) r = a[k];
  return r;
}
__device__ __forceinline__ void set8(double (&a)[8], unsigned i, double x) {
#pragma unroll
  for (unsigned k = 0; k < 8; ++k)
    if (i == k) a[k] = x;
}

// x = G^-1 rhs for one lane group (Xs = G^-1 rows in shared memory); with FP32
// factors (refine) sweeps of iterative refinement on the FP64 residual
// rhs - (x - hr0 J x), J the FP64 Jacobian rows Js.
template <typename LUT, int W>
__device__ __noinline__ double solve_ol(const LUT* Xs, const double* Js, double rhs, double hr0, int n, int lane,
                                        unsigned gm, int refine) {
  const int ld = row_ld(n);
  const bool al = lane < n;
  double xv = rowdot_ol<LUT, W>(Xs, rhs, n, ld, lane, gm);
  for (int it = 0; it < refine; ++it) {
    const double s = rowdot_ol<double, W>(Js, xv, n, ld, lane, gm);
    const double res = al ? rhs - (xv - hr0 * s) : 0.;
    xv += rowdot_ol<LUT, W>(Xs, res, n, ld, lane, gm);
  }
  return al ? xv : 0.;
}

// Candidate step scales of NewOrderNewH (MultiValueSolver.hpp:1042-1105) for
// orders p-1, p, p+1 from the last three Nordsieck differences; out of line.
struct HCand {
  double hMinus, hC, hPlus, alfa1, alfa3;
};
template <int W>
__device__ __noinline__ HCand order_candidates(double vp, double vp1, double vp2, double eps, bool al, int n,
                                               unsigned gm, unsigned p, bool try_lower, bool try_higher,
                                               double a2m, double a2p, double a2h) {
  HCand c{0., 0., 0., 0., 0.};
  if (try_lower) {
    double hm = c_gear_r.Ep[p - 1] * wrms_ol<W>(vp, eps, al, n, gm) + kMachEpsFloat;
    hm = 1. / hm;
    c.alfa1 = a2m - .05;
    c.hMinus = c.alfa1 * pow(hm, 1. / double(p));
  }
  double hc = c_gear_r.Ep[p] * wrms_ol<W>(vp1, eps, al, n, gm) + kMachEpsFloat;
  hc = 1. / hc;
  c.hC = a2p * pow(hc, 1. / double(p + 1));
  if (try_higher) {
    double hp = c_gear_r.Ep[p + 1] * wrms_ol<W>(vp2, eps, al, n, gm) + kMachEpsFloat;
    hp = 1. / hp;
    c.alfa3 = a2h - .25;
    c.hPlus = c.alfa3 * pow(hp, 1. / double(p + 2));
  }
  return c;
}

// Buffers of the round scheme.
struct RoundBufs {
  double* rec;      // [capacity][RS] cell records
  RecLayout L;
  int* act0;        // active lists (round parity 0 / 1)
  int* act1;
  int* nact;        // [2] list lengths
  unsigned char* bin;   // [capacity] bin of each list entry (compaction)
  int* bcnt;        // [kBins + 1] entries per bin
  int* bcur;        // [kBins + 1] append cursors per bin
  int* rq;          // RHS work counter: warps take the next 32 list entries from it
  int* njac;        // [2] leading Jacobian-bin entries of each list
  double* fsc;      // column scratch of the RHS threads, n words x (RHS grid threads)
  const double* rho;   // per-cell density of the constant-volume reactor, or nullptr (constant pressure)
};

}  // namespace

// ---------------------------------------------------------------------------
// init: gather, clip, renormalise (chemistry_DI.H:100-129), solver reset
// (MultiValueSolver.hpp:367-420); cells at or below tmin_chem finish here.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kAT) rounds_init_kernel(int NC, StepOptions o, StepArgs a, RoundBufs B) {
  const int n = NC + 1;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    B.nact[0] = (int)a.ncells;
    B.nact[1] = 0;
    B.njac[0] = 0;
    B.njac[1] = 0;
    *B.rq = 0;
  }
  for (long cell = (long)blockIdx.x * blockDim.x + threadIdx.x; cell < a.ncells;
       cell += (long)gridDim.x * blockDim.x) {
    B.act0[cell] = (int)cell;
    double* R = B.rec + cell * B.L.RS;
    int* RI = (int*)(R + ND_);
    const double Tc = a.T[cell];
    if (!(Tc > o.tmin_chem)) {
      double s = 0.;
      for (int i = 0; i < NC; ++i) s += a.Y[(long)i * a.ld + cell];
      for (int i = 0; i < NC; ++i) a.Y[(long)i * a.ld + cell] /= s;
      if (a.status) a.status[cell] = 0;
      if (a.nsteps) a.nsteps[cell] = 0;
      if (a.counters)
        for (int k = 0; k < NCNT; ++k) a.counters[cell * NCNT + k] = 0;
      RI[I_PHASE] = PH_DONE;
      continue;
    }
    double* va = R + B.L.ova;
    double s = 0.;
    for (int i = 0; i < NC; ++i) {
      double yi = a.Y[(long)i * a.ld + cell];
      if (yi < 0.) yi = 0.;
      va[i] = yi;
      s += yi;
    }
    for (int i = 0; i < NC; ++i) va[i] /= s;
    va[NC] = Tc;
    const double t0 = a.t0;
    R[D_T] = t0; R[D_T0] = t0; R[D_TOUT] = t0; R[D_TMESH] = t0; R[D_TSTAB] = t0;
    R[D_H] = 0.; R[D_HNEXT] = 0.; R[D_HNORD] = 0.; R[D_HSCALE] = 0.; R[D_HSCALEMAX] = 1000.;
    R[D_A24] = o.alfa2_4; R[D_A25] = o.alfa2_5; R[D_QR] = 0.; R[D_OLDCC] = 0.; R[D_HF] = 0.; R[D_HJ] = 0.;
    R[D_PENDHS] = 0.; R[D_HR0] = 0.;
    unsigned mij = 20u + 5u * (unsigned)(n - 3);
    if (mij > 50u && n < 80) mij = 50u;
    RI[I_PHASE] = PH_INIT; RI[I_STATUS] = 1; RI[I_P] = 1; RI[I_ITORDER] = 0; RI[I_ORDNEXT] = 1;
    RI[I_MAXITJ] = (int)mij; RI[I_HSTAT] = 1; RI[I_OSTAT] = 1; RI[I_FACTORIZED] = 0; RI[I_JACCHANGE] = 1;
    RI[I_CONVOK] = 1; RI[I_NSTEPS] = 0; RI[I_ITCONV] = 0; RI[I_ITCONVRATE] = 0; RI[I_ITCONVFAIL] = 0;
    RI[I_ITERRFAIL] = 0; RI[I_NCFOM] = 0; RI[I_STEPLASTJ] = 0; RI[I_ITCONST] = 0; RI[I_ITMINORD] = 0;
    RI[I_FIXEDMIN] = 0; RI[I_NEWTONK] = 0; RI[I_JCOL] = 0; RI[I_MAXORD] = o.maximum_order;
    for (int k = 0; k < NCNT; ++k) RI[I_CNT0 + k] = 0;
  }
}

// One column j of a cell's finite-difference Jacobian (KernelDense::
// NumericalJacobian, constrained branch, KernelDense.hpp:111-193):
// J(:, j) = (f(vb + hJ_j e_j) - f0) / hJ_j, stored in FP32 in the cell record.
// The n columns of a cell run on n threads of the same RHS launch; fp is this
// thread's n-word scratch (stride fs).  The T column, the reference's last,
// leaves its f in the record and sets QR, as the last evaluation did there;
// column 0 counts the n evaluations.  Out of line, so that the RHS kernel
// keeps the register budget of its single-evaluation path.
__device__ __noinline__ void jacobian_column(const MechLayout* L, const double* Md, const int* Mi, double* scratch,
                                             double* R, const RecLayout RL, int j, double P0, int energy,
                                             double y_max_T, double* fp, long fs, double rho0) {
  const int n = L->nc + 1;
  const double* vb = R + RL.ovb;
  const double yh = vb[j], ej = R[RL.oeps + j];
  const double hf = R[D_HF];
  const double aa = fabs(yh), bb = fabs(1. / ej);
  double hJ = sqrt(kMachEpsDouble) * (aa > bb ? aa : bb);
  hJ = fmax(hJ, hf / ej);
  hJ = fmax(hJ, sqrt(kTinyFloat));
  if (yh + hJ > (j < n - 1 ? 1. : y_max_T)) hJ = -hJ;
  const bool last = j == n - 1;
  double* f = last ? R + RL.of : fp;
  const long ffs = last ? 1 : fs;
  const double q = rhs_cell(L, Md, Mi, scratch, vb, 1, j, yh + hJ, f, ffs, P0, energy, rho0);
  const double* f0 = R + RL.of0;
  double* Jg = R + RL.ojac;
  const double hInv = 1. / hJ;
  for (int i = 0; i < n; ++i) Jg[i * n + j] = hInv * (f[(long)i * ffs] - f0[i]);
  if (last) R[D_QR] = q;
  if (j == 0) {
    int* RI = (int*)(R + ND_);
    RI[I_CNT0 + CNT_JAC_RHS] += n;
  }
}

// ---------------------------------------------------------------------------
// rhs: one thread per requested evaluation.  The list starts with the cells
// that build a Jacobian (njac of them, the compaction's first bin); each of
// those is n work items, one per column, the other cells one item each.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kRT, 4) rounds_rhs_kernel(MechLayout Lp, const unsigned char* __restrict__ mech_gmem,
                                                          int energy, double P0, double y_max_T, RoundBufs B, int par,
                                                          int analytic, int* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ MechLayout sL;
  if (threadIdx.x == 0) sL = Lp;
  if (blockIdx.x == 0 && threadIdx.x < 2 * (kBins + 1)) {   // this round's compaction counts from zero
    if (threadIdx.x < kBins + 1) B.bcnt[threadIdx.x] = 0;
    else B.bcur[threadIdx.x - kBins - 1] = 0;
  }
  if (!stage_bulk(smem, mech_gmem, Lp.bytes, &mbar, err)) return;
  const double* Md = (const double*)smem;
  const int* Mi = (const int*)(smem + (size_t)Lp.n_double * sizeof(double));
  double* scratch = (double*)(smem + ((Lp.bytes + 15u) & ~15u));
  const RecLayout RL = B.L;
  const int nact = B.nact[par];
  const int njac = B.njac[par];
  const int n = Lp.nc + 1;
  const int* act = par ? B.act1 : B.act0;
  // items per Jacobian cell: its n columns by forward differences, or (analytic) the species columns
  // as one item and the temperature column (a forward difference) as another
  const int jitems = analytic ? 2 : n;
  const int nitems = njac * jitems + (nact - njac);
  double* fp = B.fsc + (long)blockIdx.x * kRT + threadIdx.x;   // this thread's column scratch
  const long fs = (long)gridDim.x * kRT;
  // Dynamic distribution: each warp takes the next 32 work items.  Consecutive items of a Jacobian are
  // consecutive columns of one cell, so a warp's J stores and record reads land on neighbouring words.
  const int wl = threadIdx.x & 31;
  for (;;) {
    int base = 0;
    if (wl == 0) base = atomicAdd(B.rq, 32);
    base = __shfl_sync(kFull, base, 0);
    if (base >= nitems) break;
    const int item = base + wl;
    if (item >= nitems) continue;
    if (item < njac * jitems) {
      const int e = item / jitems;
      const int cell = act[e];
      double* R = B.rec + (long)cell * RL.RS;
      const int col = item - e * jitems;
      if (!analytic) {
        jacobian_column(&sL, Md, Mi, scratch, R, RL, col, P0, energy, y_max_T, fp, fs, B.rho ? B.rho[cell] : 0.);
      } else if (col == 0) {
        analytic_jacobian_species(&sL, Md, Mi, scratch, R + RL.ovb, 1, P0, energy, R + RL.ojac);
      } else {
        jacobian_column(&sL, Md, Mi, scratch, R, RL, n - 1, P0, energy, y_max_T, fp, fs, 0.);
        int* RI = (int*)(R + ND_);
        RI[I_CNT0 + CNT_JAC_RHS] += 1;
      }
      continue;
    }
    const int cell = act[njac + (item - njac * jitems)];
    double* R = B.rec + (long)cell * RL.RS;
    int* RI = (int*)(R + ND_);
    const int ph = RI[I_PHASE];
    if (!rhs_phase(ph)) continue;
    if (ph == PH_JAC) {   // a Jacobian outside the list head (not produced by the compaction): serially
      if (analytic) {
        analytic_jacobian_species(&sL, Md, Mi, scratch, R + RL.ovb, 1, P0, energy, R + RL.ojac);
        jacobian_column(&sL, Md, Mi, scratch, R, RL, n - 1, P0, energy, y_max_T, fp, fs, 0.);
        RI[I_CNT0 + CNT_JAC_RHS] += 1;
      } else {
        for (int j = 0; j < n; ++j)
          jacobian_column(&sL, Md, Mi, scratch, R, RL, j, P0, energy, y_max_T, fp, fs, B.rho ? B.rho[cell] : 0.);
      }
      continue;
    }
    const double* src = R + RL.ova;
    double* dst = R + RL.of;
    int pj = -1;
    double pval = 0.;
    if (ph == PH_PRED) {
      src = R + RL.ovb;
      dst = R + RL.of0;
    } else if (ph == PH_STAB_CONV || ph == PH_STAB_ERR) {
      src = R + RL.oz;
    }
    R[D_QR] = rhs_cell(&sL, Md, Mi, scratch, src, 1, pj, pval, dst, 1, P0, energy, B.rho ? B.rho[cell] : 0.);
    RI[I_CNT0 + CNT_RHS] += 1;
  }
}

// ---------------------------------------------------------------------------
// Source terms and diagonal Jacobian of the steady solvers (laminarSMOKE
// steady/linearModel.H:92-170 as jacobianEvaluation.H:60-92 calls it), one
// thread per cell:
//   S_i = R_i MW_i (i < NC), S_NC = QR at omega = max(Y, 0), T and the cell's
//   pressure;
//   J_k = (S_k(y + dy_k e_k) - S_k(y)) / dy_k with the increment dy_k of
//   reactionJacobian (:132-170), the perturbed mass fraction clipped at zero
//   as reactionSourceTerms clips it;
//   implicit_k = J_k, explicit_k = S_k - J_k y_k (y unclipped).
// yb, s0, sp: scratch [n][ncells] (clipped state, S(y), S(y + dy e_k)).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kRT, 4) steady_sources_kernel(MechLayout Lp, const unsigned char* __restrict__ mech_gmem,
                                                                long ncells, const double* __restrict__ Y,
                                                                const double* __restrict__ T, long ld,
                                                                const double* __restrict__ pc, double p_scalar,
                                                                double* __restrict__ yb, double* __restrict__ s0,
                                                                double* __restrict__ sp, double* __restrict__ Simp,
                                                                double* __restrict__ Sexp, long lds, int* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ MechLayout sL;
  if (threadIdx.x == 0) sL = Lp;
  if (!stage_bulk(smem, mech_gmem, Lp.bytes, &mbar, err)) return;
  const double* Md = (const double*)smem;
  const int* Mi = (const int*)(smem + (size_t)Lp.n_double * sizeof(double));
  double* scratch = (double*)(smem + ((Lp.bytes + 15u) & ~15u));
  const int NC = Lp.nc, n = NC + 1;
  const double ZERO_DER = sqrt(kTinyFloat);
  const double ETA2 = sqrt(kMachEpsDouble);
  const double TOLR = 1.e-7, TOLA = 1.e-12;
  for (long c = (long)blockIdx.x * kRT + threadIdx.x; c < ncells; c += (long)gridDim.x * kRT) {
    for (int i = 0; i < NC; ++i) yb[(long)i * ncells + c] = fmax(Y[(long)i * ld + c], 0.);
    yb[(long)NC * ncells + c] = T[c];
    const double P0 = pc ? pc[c] : p_scalar;
    const double* y = yb + c;
    s0[(long)NC * ncells + c] = rhs_cell<true>(&sL, Md, Mi, scratch, y, ncells, -1, 0., s0 + c, ncells, P0, 1, 0.);
    for (int k = 0; k < n; ++k) {
      const double yk = k < NC ? Y[(long)k * ld + c] : T[c];
      const double ew = 1. / (TOLA + TOLR * fabs(yk));
      double hJ = ETA2 * fabs(fmax(yk, 1. / ew));
      const double hJf = 1. / ew;
      hJ = fmax(hJ, hJf);
      hJ = fmax(hJ, ZERO_DER);
      const double dy = fmin(hJ, 1.e-3 + 1e-3 * fabs(yk));
      const double udy = 1. / dy;
      double pv = yk + dy;
      if (k < NC) pv = fmax(pv, 0.);
      const double qp = rhs_cell<true>(&sL, Md, Mi, scratch, y, ncells, k, pv, sp + c, ncells, P0, 1, 0.);
      const double spk = k < NC ? sp[(long)k * ncells + c] : qp;
      const double s0k = s0[(long)k * ncells + c];
      const double J = (spk - s0k) * udy;
      Simp[(long)k * lds + c] = J;
      Sexp[(long)k * lds + c] = s0k - J * yk;
    }
  }
}

// Fall-off correction of slot fo at the third-body concentration Mc (KineticsMap_CHEMKIN.hpp:1552-1610,
// FallOffReactionsCorrection): k_inf (Pr / (1 + Pr)) F / kArr.
__device__ __forceinline__ double falloff_corr(const MechView& M, const MechLayout& L, int fo, double kArr, double Mc,
                                              double T, double logT, double uT) {
  const double kInf = exp(M.D(L.fo_lnA)[fo] + M.D(L.fo_beta)[fo] * logT - M.D(L.fo_eor)[fo] * uT);
  const double a = M.D(L.fo_a)[fo], b = M.D(L.fo_b)[fo], c = M.D(L.fo_c)[fo], d = M.D(L.fo_d)[fo];
  const int ty = M.I(L.fo_type)[fo];
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
    double xSRI = 0.;
    if (Pr > 1.e-32) {
      const double l10 = log10(Pr);
      xSRI = 1. / (1. + l10 * l10);
    }
    wF = pow(lF, xSRI) * d;
    const double e = M.D(L.fo_e)[fo];
    if (e != 0.) wF *= pow(T, e);
  }
  return kInf * (Pr / (1. + Pr)) * wF / kArr;
}

// ---------------------------------------------------------------------------
// The steady solvers' default linearisation (sparseJacobian true,
// steady/readOptionsSteadyState.H:46): linearModel::reactionJacobianSparse
// (steady/linearModel.H:172-232).  The species entries of the diagonal are
// JacobianSparsityPatternMap::Jacobian (maps/JacobianSparsityPatternMap.hpp:
// 427-560) at omega* = max(max(Y, 0), 1e-13), times MW:
//   J_k = MW_k sum_j nu_kj [ lambda_jk r_f,j / omega*_k - nu'_jk r_b,j / omega*_k
//         + (r_f,j - r_b,j) c*_k / omega*_k (eps_jk - 1) / M_j              (third body)
//         + (r_f,j - r_b,j) dG_jk / G_j   or  (r_f,j - r_b,j)  (fall-off / CABR) ]
// each term present where the reaction's orders, products, efficiencies or
// bath name k; dG a forward difference of the fall-off correction with an
// omega increment of 1e-4, at fixed density; the kinetics evaluated at
// c* = omega* rho* / MW with cTot = P / (R T) given.  Thread-serial; scratch
// as rhs_cell: C = c*, G = h/RT - s/R, R = the accumulated diagonal.  Y: the
// unclipped mass fractions (stride ys).  Writes J_k to Jk[k * js].
// ---------------------------------------------------------------------------
__device__ __noinline__ void steady_sparse_diagonal(const MechLayout* __restrict__ Lp, const double* __restrict__ Md,
                                                    const int* __restrict__ Mi, double* __restrict__ scratch,
                                                    const double* __restrict__ Yc, long ys, double T, double P0,
                                                    double* __restrict__ Jk, long js) {
  const MechLayout& L = *Lp;
  const MechView M{Md, Mi};
  const int NC = L.nc, NR = L.nr;
  const int tid = threadIdx.x;
  double* C = scratch;
  double* G = scratch + NC * kRT;
  double* D = scratch + 2 * NC * kRT;
#define SC_(arr, i) arr[(i) * kRT + tid]
  const double* MW = M.D(L.mw);
  const double eps = 1.e-13;
  auto om = [&](int k) {
    const double o = fmax(Yc[(long)k * ys], 0.);
    return o > eps ? o : eps;
  };
  double u = 0.;
  for (int i = 0; i < NC; ++i) u += om(i) / MW[i];
  const double MWs = 1. / u;
  const double cTs = P0 / kRgas / T;
  const double rhos = cTs * MWs;
  const double* TM = M.D(L.t_mid);
  const double T2 = T * T, T3 = T2 * T, T4 = T3 * T, uT = 1. / T;
  const double logT = log(T);
  const double lP = log(101325. / kRgas / T);
  for (int i = 0; i < NC; ++i) {
    SC_(C, i) = om(i) * rhos / MW[i];
    const bool hi = T > TM[i];
    const double* A = hi ? M.D(L.dh_ht) + 6 * i : M.D(L.dh_lt) + 6 * i;
    const double hrt = A[0] + T * A[1] + T2 * A[2] + T3 * A[3] + T4 * A[4] + uT * A[5];
    const double* B = hi ? M.D(L.ds_ht) + 6 * i : M.D(L.ds_lt) + 6 * i;
    SC_(G, i) = hrt - (B[0] * logT + T * B[1] + T2 * B[2] + T3 * B[3] + T4 * B[4] + B[5]);
    SC_(D, i) = 0.;
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
  const int* op = M.I(L.ford_ptr);
  const int* osp = M.I(L.ford_sp);
  const double* onu = M.D(L.ford_val);
  const int* pp = M.I(L.prod_ptr);
  const int* psp = M.I(L.prod_sp);
  const double* pnu = M.D(L.prod_nu);
  for (int j = 0; j < NR; ++j) {
    double kArr = exp(lnA[j] + beta[j] * logT - eor[j] * uT);
    if (sgn[j] < 0) kArr *= -1.;
    if (L.n_plog > 0) {
      const int ps = M.I(L.plog_slot)[j];
      if (ps >= 0) kArr = plog_k(M, L, ps, T, logT, P0);
    }
    if (L.n_cheb > 0) {
      const int cs = M.I(L.cheb_slot)[j];
      if (cs >= 0) kArr = cheb_k(M, L, cs, T, P0);
    }
    if (L.n_xplog > 0) {
      const int xs = M.I(L.xplog_slot)[j];
      if (xs >= 0) kArr = xplog_k(M, L, xs, T, logT, P0, cTs, [&](int k) { return SC_(C, k); });
    }
    double kMod = kArr, Mtb = 0.;
    const int tb = tbs[j];
    if (tb >= 0) {
      Mtb = cTs;
      const int* tp = M.I(L.tb_ptr);
      const int* ts = M.I(L.tb_sp);
      const double* te = M.D(L.tb_eff);
      for (int q = tp[tb]; q < tp[tb + 1]; ++q) Mtb += SC_(C, ts[q]) * te[q];
      kMod *= Mtb;
    }
    const int fo = fos[j];
    bool cabr = false;
    double Gcorr = 1.;
    if (fo >= 0) {
      cabr = M.I(L.fo_cabr)[fo] != 0;
      const int single = M.I(L.fo_single)[fo];
      double Mc;
      if (single < 0) {
        Mc = cTs;
        const int* fp = M.I(L.fo_ptr);
        const int* fs = M.I(L.fo_sp);
        const double* fe = M.D(L.fo_eff);
        for (int q = fp[fo]; q < fp[fo + 1]; ++q) Mc += SC_(C, fs[q]) * fe[q];
      } else {
        Mc = SC_(C, single) + 1.e-16;
      }
      if (cabr) {
        // KineticsMap_CHEMKIN::ChemicallyActivatedBimolecularReactions (:1613-1660): F / (1 + Pr)
        const double kInf = exp(M.D(L.fo_lnA)[fo] + M.D(L.fo_beta)[fo] * logT - M.D(L.fo_eor)[fo] * uT);
        const double Pr = kArr * Mc / kInf;
        const double a = M.D(L.fo_a)[fo], b = M.D(L.fo_b)[fo], c = M.D(L.fo_c)[fo], d = M.D(L.fo_d)[fo];
        const int ty = M.I(L.fo_type)[fo];
        double wF = 1.;
        if (ty == 1) {
          double v = (1. - a) * exp(-T / b) + a * exp(-T / c);
          if (d != 0.) v += exp(-d / T);
          const double lF = (v < 1.e-300) ? -300. : log10(v);
          const double nTroe = 0.75 - 1.27 * lF;
          const double cTroe = -0.4 - 0.67 * lF;
          const double sTroe = log10(Pr) + cTroe;
          const double qq = sTroe / (nTroe - 0.14 * sTroe);
          wF = exp10(lF / (1. + qq * qq));
        } else if (ty == 2) {
          const double lF = a * exp(-b / T) + exp(-T / c);
          const double l10 = log10(Pr);
          wF = pow(lF, 1. / (1. + l10 * l10)) * d;
          const double e = M.D(L.fo_e)[fo];
          if (e != 0.) wF *= pow(T, e);
        }
        kMod *= (1. / (1. + Pr)) * wF;
      } else {
        Gcorr = falloff_corr(M, L, fo, kArr, Mc, T, logT, uT);
        kMod *= Gcorr;
      }
    }
    if (L.n_xfo > 0) {    // extended fall-off (KineticsMap_CHEMKIN.hpp:1672-1681)
      const int xs = M.I(L.xfo_slot)[j];
      if (xs >= 0) {
        kArr = xfo_k(M, L, xs, T, cTs, [&](int k) { return SC_(C, k); });
        kMod = kArr;
      }
    }
    double fwd = 1.;
    for (int q = op[j]; q < op[j + 1]; ++q) fwd *= conc_factor_r(onu[q], SC_(C, osp[q]));
    double rbj = 0.;
    const int kind = rk[j];
    if (kind != 0) {
      double rv = 1.;
      for (int q = pp[j]; q < pp[j + 1]; ++q) rv *= conc_factor_r(pnu[q], SC_(C, psp[q]));
      double rf;
      if (kind == 1) {
        double dg = 0.;
        for (int q = pp[j]; q < pp[j + 1]; ++q) dg += contrib_r(pnu[q], SC_(G, psp[q]));
        for (int q = rp[j]; q < rp[j + 1]; ++q) dg -= contrib_r(rnu[q], SC_(G, rsp[q]));
        rf = exp(dg - lP * dnu[j]);
      } else {
        const int sr = rs[j];
        rf = exp(M.D(L.rev_lnA)[sr] + M.D(L.rev_beta)[sr] * logT - M.D(L.rev_eor)[sr] * uT) / kArr;
      }
      rbj = (rv * rf) * kMod;
    }
    const double rfj = kMod * fwd;
    // the bracket of species k in reaction j
    auto bracket = [&](int k) {
      const double omk = om(k);
      double v = 0.;
      for (int q = op[j]; q < op[j + 1]; ++q)
        if (osp[q] == k) v = onu[q] * rfj / omk;
      for (int q = pp[j]; q < pp[j + 1]; ++q)
        if (psp[q] == k) v -= pnu[q] * rbj / omk;
      if (tb >= 0) {
        const int* tp = M.I(L.tb_ptr);
        const int* ts = M.I(L.tb_sp);
        const double* te = M.D(L.tb_eff);
        for (int q = tp[tb]; q < tp[tb + 1]; ++q)
          if (ts[q] == k) v += (rfj - rbj) * SC_(C, k) / omk * te[q] / Mtb;
      }
      if (fo >= 0) {
        const int single = M.I(L.fo_single)[fo];
        bool has = single == k;
        const int* fp = M.I(L.fo_ptr);
        const int* fs = M.I(L.fo_sp);
        const double* fe = M.D(L.fo_eff);
        if (single < 0)
          for (int q = fp[fo]; q < fp[fo + 1]; ++q)
            if (fs[q] == k) has = true;
        if (has) {
          if (cabr) {
            v += (rfj - rbj);
          } else {
            // M at c* with c*_k from omega*_k + 1e-4 (density unchanged)
            const double ck_plus = (omk + 1.e-4) * rhos / MW[k];
            double Mp;
            if (single < 0) {
              Mp = cTs;
              for (int q = fp[fo]; q < fp[fo + 1]; ++q) Mp += (fs[q] == k ? ck_plus : SC_(C, fs[q])) * fe[q];
            } else {
              Mp = ck_plus + 1.e-16;
            }
            const double Gp = falloff_corr(M, L, fo, kArr, Mp, T, logT, uT);
            const double dG = (Gp - Gcorr) / 1.e-4;
            v += (rfj - rbj) * dG / Gcorr;
          }
        }
      }
      return v;
    };
    for (int q = rp[j]; q < rp[j + 1]; ++q) SC_(D, rsp[q]) -= rnu[q] * bracket(rsp[q]);
    for (int q = pp[j]; q < pp[j + 1]; ++q) SC_(D, psp[q]) += pnu[q] * bracket(psp[q]);
  }
  for (int k = 0; k < NC; ++k) Jk[(long)k * js] = SC_(D, k) * MW[k];
#undef SC_
}

// sparseJacobian true: the species diagonal of steady_sparse_diagonal (with speciesEquations on, else
// zero) and the temperature entry by the forward difference of the dense path (with energyEquation on,
// else zero).  yb, s0, sp: scratch [n][ncells].
__global__ void __launch_bounds__(kRT, 4) steady_sources_sparse_kernel(
    MechLayout Lp, const unsigned char* __restrict__ mech_gmem, long ncells, const double* __restrict__ Y,
    const double* __restrict__ T, long ld, const double* __restrict__ pc, double p_scalar, int species, int energy,
    double* __restrict__ yb, double* __restrict__ s0, double* __restrict__ sp, double* __restrict__ Simp,
    double* __restrict__ Sexp, long lds, int* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ MechLayout sL;
  if (threadIdx.x == 0) sL = Lp;
  if (!stage_bulk(smem, mech_gmem, Lp.bytes, &mbar, err)) return;
  const double* Md = (const double*)smem;
  const int* Mi = (const int*)(smem + (size_t)Lp.n_double * sizeof(double));
  double* scratch = (double*)(smem + ((Lp.bytes + 15u) & ~15u));
  const int NC = Lp.nc, n = NC + 1;
  for (long c = (long)blockIdx.x * kRT + threadIdx.x; c < ncells; c += (long)gridDim.x * kRT) {
    for (int i = 0; i < NC; ++i) yb[(long)i * ncells + c] = fmax(Y[(long)i * ld + c], 0.);
    yb[(long)NC * ncells + c] = T[c];
    const double P0 = pc ? pc[c] : p_scalar;
    const double* y = yb + c;
    s0[(long)NC * ncells + c] = rhs_cell<true>(&sL, Md, Mi, scratch, y, ncells, -1, 0., s0 + c, ncells, P0, 1, 0.);
    double JT = 0.;
    if (energy) {   // linearModel.H:195-230, the dense path's increment for the T entry
      const double yk = T[c];
      const double ew = 1. / (1.e-12 + 1.e-7 * fabs(yk));
      double hJ = sqrt(kMachEpsDouble) * fabs(fmax(yk, 1. / ew));
      hJ = fmax(hJ, 1. / ew);
      hJ = fmax(hJ, sqrt(kTinyFloat));
      const double dy = fmin(hJ, 1.e-3 + 1e-3 * fabs(yk));
      const double qp = rhs_cell<true>(&sL, Md, Mi, scratch, y, ncells, NC, yk + dy, sp + c, ncells, P0, 1, 0.);
      JT = (qp - s0[(long)NC * ncells + c]) * (1. / dy);
    }
    if (species) {
      steady_sparse_diagonal(&sL, Md, Mi, scratch, Y + c, ld, T[c], P0, Simp + c, lds);
    } else {
      for (int k = 0; k < NC; ++k) Simp[(long)k * lds + c] = 0.;
    }
    Simp[(long)NC * lds + c] = JT;
    for (int k = 0; k < n; ++k) {
      const double yk = k < NC ? Y[(long)k * ld + c] : T[c];
      Sexp[(long)k * lds + c] = s0[(long)k * ncells + c] - Simp[(long)k * lds + c] * yk;
    }
  }
}

// ---------------------------------------------------------------------------
// advance: one lane group per listed cell -- a warp, or half a warp when the
// cell has at most 16 components (two cells per warp) -- lane k of the group
// holds component k of every vector.  Consumes the RHS result and runs the solver to its next request.
// ---------------------------------------------------------------------------
template <typename LUT, int W>
__global__ void __launch_bounds__(kWA * 32, 4) rounds_advance_kernel(int NC, StepOptions o, StepArgs a, RoundBufs B,
                                                                      int par) {
  extern __shared__ __align__(16) unsigned char wsm[];
  constexpr int CPW = 32 / W;   // cells per warp
  const int wl = threadIdx.x & 31;
  const int lane = wl & (W - 1);                     // component owned by this thread
  const int w = (threadIdx.x >> 5) * CPW + wl / W;   // lane group within the block
  const unsigned gm = W == 32 ? kFull : (0xffffu << (wl & 16));
  const int n = NC + 1, ld = row_ld(n);
  const RecLayout RL = B.L;
  // per-warp shared memory: G^-1 X[n][ld] (LUT), the Gauss-Jordan work array A[n][2n+1] (LUT), its pivot
  // row K[2n] (LUT) and the Jacobian J[n][ld] (double)
  const int la = 2 * n + 1;
  constexpr int G = kWA * CPW;   // lane groups per block
  LUT* Xs = (LUT*)wsm + (size_t)w * n * ld;
  LUT* As = (LUT*)wsm + (size_t)G * n * ld + (size_t)w * n * la;
  LUT* Ks = (LUT*)wsm + (size_t)G * n * ld + (size_t)G * n * la + (size_t)w * 2 * n;
  double* Js = (double*)((LUT*)wsm + (((size_t)G * (n * ld + n * la + 2 * n) + 1) & ~(size_t)1)) + (size_t)w * n * ld;
  const bool al = lane < n;
  const double lo = lane < NC ? 0. : o.y_min_T, hi = lane < NC ? 1. : o.y_max_T;
  const int nact = B.nact[par];
  const int* act = par ? B.act1 : B.act0;
  for (int widx = blockIdx.x * G + w; widx < nact; widx += gridDim.x * G) {
    const int cell = act[widx];
    double* R = B.rec + (long)cell * RL.RS;
    int* RI = (int*)(R + ND_);
    {
      // ask L2 for the record this group visits next, so its DRAM latency overlaps this visit
      const int wn = widx + gridDim.x * G;
      if (wn < nact) {
        const char* Rn = (const char*)(B.rec + (long)act[wn] * RL.RS);
        for (int off = lane * 128; off < RL.RS * 8; off += W * 128)
          asm volatile("prefetch.global.L2 [%0];" ::"l"(Rn + off));
      }
    }
    int phase = RI[I_PHASE];
    if (!rhs_phase(phase)) continue;   // same in all lanes
    // ---- scalar state (every lane reads the same words) ----
    double t = R[D_T];
    const double t0 = R[D_T0];
    double tOut = R[D_TOUT], tInMeshPoint = R[D_TMESH], tStabilize = R[D_TSTAB], h = R[D_H];
    double hNextStep = R[D_HNEXT], hNordsieck = R[D_HNORD], hScale = R[D_HSCALE], hScaleMax = R[D_HSCALEMAX];
    double alfa2_4 = R[D_A24], alfa2_5 = R[D_A25], oldCC = R[D_OLDCC];
    const double QR = R[D_QR];
    double hf = R[D_HF], hJ = R[D_HJ], pendHScale = R[D_PENDHS], hr0f = R[D_HR0];
    int status = RI[I_STATUS];
    unsigned p = RI[I_P], iterOrder = RI[I_ITORDER], orderInNextStep = RI[I_ORDNEXT];
    const unsigned maxIterationsJacobian = RI[I_MAXITJ];
    int odeHStatus = RI[I_HSTAT], odeOrderStatus = RI[I_OSTAT], factorized = RI[I_FACTORIZED];
    int jacobianChange = RI[I_JACCHANGE], convOK = RI[I_CONVOK];
    unsigned numberOfSteps = RI[I_NSTEPS], iterConvergence = RI[I_ITCONV];
    unsigned iterConvergenceRate = RI[I_ITCONVRATE], iterConvergenceFailure = RI[I_ITCONVFAIL];
    unsigned iterErrorFailure = RI[I_ITERRFAIL], nConvFailOrderMax = RI[I_NCFOM];
    unsigned stepOfLastJacobian = RI[I_STEPLASTJ], iterConstSteps = RI[I_ITCONST];
    unsigned iterMinimumOrder = RI[I_ITMINORD];
    bool fixedOrderMin = RI[I_FIXEDMIN] != 0;
    unsigned newtonK = RI[I_NEWTONK];
    int jcol = RI[I_JCOL];
    unsigned maximum_order = RI[I_MAXORD];
    int cstep = 0, csolve = 0, cjac = 0, cfact = 0, cerr = 0, cconv = 0;
    // ---- vectors, one component per lane ----
    double z[8], v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      z[i] = al ? R[RL.oz + i * n + lane] : 0.;
      v[i] = al ? R[RL.ov + i * n + lane] : 0.;
    }
    double b = al ? R[RL.ob + lane] : 0., f = al ? R[RL.of + lane] : 0., f0 = al ? R[RL.of0 + lane] : 0.;
    double va = al ? R[RL.ova + lane] : 0., vb = al ? R[RL.ovb + lane] : 0., eps = al ? R[RL.oeps + lane] : 0.;
    double x = 0.;                 // latest Newton correction
    bool dz = false, dv = false;   // z / v modified
    bool j_in = false, inv_in = false;
    double* const Jg = R + RL.ojac;
    LUT* const Ig = (LUT*)(R + RL.oinv);
    // Rounds that solve (predictor and Newton results) will want G^-1 and, for the refinement and the
    // convergence-rate test, J: start copying this lane's rows into shared memory now.
    bool pending = false;
    if (phase == PH_PRED || phase == PH_NEWTON) {
      if (al)
        for (int j = 0; j < n; ++j) {
          cp_async_el(&Xs[lane * ld + j], &Ig[lane * n + j]);
          cp_async8(&Js[lane * ld + j], &Jg[lane * n + j]);
        }
      pending = true;
    }
    auto drain = [&]() {
      if (pending) {
        cp_async_wait_all();
        __syncwarp(gm);
        pending = false;
        inv_in = j_in = true;
      }
    };

    enum : int { H_DEC = 0, H_CONST = 1, H_INC = 2 };
    enum : int { O_DEC = 0, O_CONST = 1, O_INC = 2 };
    auto alfa2 = [&](unsigned k) { return k == 4 ? alfa2_4 : (k == 5 ? alfa2_5 : .8); };
    auto wrms = [&](double xv) { return wrms_ol<W>(xv, eps, al, n, gm); };
    auto clamp = [&](double y) {
      if (al) {
        if (y < lo) y = lo;
        if (y > hi) y = hi;
      }
      return y;
    };
    auto load_j = [&]() {   // this cell's Jacobian rows into shared memory
      drain();
      if (!j_in) {
        if (al)
          for (int j = 0; j < n; ++j) Js[lane * ld + j] = Jg[lane * n + j];
        __syncwarp(gm);
        j_in = true;
      }
    };
    auto load_inv = [&]() {
      drain();
      if (!inv_in) {
        if (al)
          for (int j = 0; j < n; ++j) Xs[lane * ld + j] = Ig[lane * n + j];
        __syncwarp(gm);
        inv_in = true;
      }
    };
    // x = G^-1 rhs; with FP32 factors refinement sweeps on the FP64 residual
    // rhs - (x - hr0 J x) of the stored FP64 Jacobian
    auto solve = [&](double rhs) {
      load_inv();
      const bool fp32 = sizeof(LUT) == sizeof(float);
      if (fp32) load_j();
      ++csolve;
      return solve_ol<LUT, W>(Xs, Js, rhs, hr0f, n, lane, gm, fp32 ? kRefineR : 0);
    };
    auto factorize = [&]() {
      load_j();
      gj_inverse<LUT, W>(Js, As, Ks, Xs, Ig, hr0f, n, lane, gm);
      inv_in = true;
      ++cfact;
    };
    auto fail_keep_z = [&](int st) {
      status = st;
      va = z[0];
    };

    enum : int { L_NONE, L_START_STEP, L_DRIVER_LOOP, L_JAC_COLUMN, L_AFTER_JAC, L_AFTER_FACT, L_NEWTON_TEST,
                 L_CORR_DONE, L_FINISH };
    int lab = L_NONE;
    switch (phase) {
      case PH_INIT: {
        // MultiValueSolver::Solve, first call (:445-469)
        const bool illegal = al && (va < lo || va > hi);
        if (__any_sync(gm, illegal)) { status = -9; lab = L_FINISH; break; }
        eps = al ? 1. / (o.atol + o.rtol * fabs(va)) : 0.;
        double lo0, hi0;
        if (t0 != 0.) { lo0 = 100. * kMachEpsDouble * fabs(t0); hi0 = fabs(t0); }
        else { lo0 = kMachEpsDouble; hi0 = 1.e-4; }
        double h0 = 0.5 / (wrms(f) + kMachEpsFloat);
        if (h0 < lo0) h0 = lo0;
        if (h0 > hi0) h0 = hi0;
        const double dtc = a.dt ? a.dt[cell] : a.dt_scalar;
        tOut = t0 + dtc;
        h0 *= fabs(tOut - t0) / (tOut - t0);
        z[0] = va;
        z[1] = f * h0;
        dz = true;
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
          hf = 1.e+3 * kMachEpsDouble * fabs(h) * wrms(f0) * double(n);
          if (hf < 1.e-10) hf = 1.;
          jcol = 0;
          lab = L_JAC_COLUMN;
          break;
        }
        lab = L_AFTER_JAC;
        break;
      }
      case PH_JAC: {
        // the RHS kernel has built every column of J
        ++cjac;
        factorized = 0;
        lab = L_AFTER_JAC;
        break;
      }
      case PH_NEWTON: {
        x = solve(al ? f * h - v[1] - b : 0.);
        b += x;
        ++newtonK;
        if (newtonK > 4u) { convOK = 0; iterConvergence = 4; lab = L_CORR_DONE; }
        else lab = L_NEWTON_TEST;
        break;
      }
      case PH_STAB_CONV: {
        z[1] = f * h;
        dz = true;
        tStabilize = tInMeshPoint;
        if (numberOfSteps > stepOfLastJacobian + 5u) jacobianChange = 1;
        if (numberOfSteps != stepOfLastJacobian && iterConvergenceFailure == 50u) jacobianChange = 1;
        hNextStep *= pendHScale;
        lab = L_DRIVER_LOOP;
        break;
      }
      case PH_STAB_ERR: {
        z[1] = f * h;
        dz = true;
        tStabilize = tInMeshPoint;
        odeHStatus = H_DEC;
        hNextStep *= hScale;
        lab = L_DRIVER_LOOP;
        break;
      }
      default:   // PH_FINAL
        lab = L_FINISH;
        break;
    }

    // labels that need no RHS; a request or a finish is reached within a few hops
    for (int hop = 0; lab != L_NONE; ++hop) {
      if (hop >= 64) {
        fail_keep_z(-10);
        lab = L_FINISH;
      }
      switch (lab) {
        case L_START_STEP: {
          // MultiValueSolver::Solve loop (:532-560) + DriverStep prologue (:753-776)
          if (numberOfSteps >= (unsigned)o.max_steps) { fail_keep_z(-1); lab = L_FINISH; break; }
          eps = al ? 1. / (o.atol + o.rtol * fabs(z[0])) : 0.;
          if (kMachEpsDouble * wrms(z[0]) > 1.) { fail_keep_z(-2); lab = L_FINISH; break; }
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
            double hr = 1.;
#pragma unroll
            for (unsigned i = 1; i < 8; ++i) {
              if (i <= p) {
                hr *= hScale;
                z[i] *= hr;
              }
            }
            z[0] = clamp(z[0]);
            dz = true;
            iterOrder = 0;
            odeHStatus = H_CONST;
          }
          h = hNextStep;
          hNordsieck = hNextStep;
          t = tInMeshPoint + h;
          if (t == tInMeshPoint) {
            fail_keep_z(-6);
            t = tInMeshPoint;
            lab = L_FINISH;
            break;
          }
          {
            // MultiValueStep prediction v = D z with min/max handling, then vb = CheckConstraints(v0)
            double wv[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) wv[i] = (i <= (int)p) ? z[i] : 0.;
#pragma unroll
            for (int i = 0; i < 7; ++i)
#pragma unroll
              for (int j = 6; j >= 0; --j)
                if (i < (int)p && j >= i && j <= (int)p - 1) wv[j] += wv[j + 1];
            if (al) {
              if (wv[0] < lo && fabs(wv[0] - lo) * eps < double(n)) {
                wv[1] = lo - z[0];
                wv[0] = lo;
#pragma unroll
                for (int i = 2; i < 8; ++i) wv[i] = 0.;
              }
              if (wv[0] > hi && fabs(wv[0] - hi) * eps < double(n)) {
                wv[1] = hi - z[0];
                wv[0] = hi;
#pragma unroll
                for (int i = 2; i < 8; ++i) wv[i] = 0.;
              }
            }
#pragma unroll
            for (int i = 0; i < 8; ++i)
              if (i <= (int)p) v[i] = wv[i];
            dv = true;
            vb = clamp(wv[0]);
          }
          phase = PH_PRED;
          lab = L_NONE;
          break;
        }
        case L_JAC_COLUMN: {
          // KernelDense::NumericalJacobian: the RHS kernel evaluates all n perturbed states next
          phase = PH_JAC;
          lab = L_NONE;
          break;
        }
        case L_AFTER_JAC: {
          if (factorized && iterOrder == 0) factorized = 0;
          if (!factorized) {
            hr0f = h * c_gear_r.r[0][p - 1];
            factorize();
            factorized = 1;
          }
          lab = L_AFTER_FACT;
          break;
        }
        case L_AFTER_FACT: {
          x = solve(al ? f0 * h - v[1] : 0.);
          b = x;
          newtonK = 1;
          lab = L_NEWTON_TEST;
          break;
        }
        case L_NEWTON_TEST: {
          const double r0 = c_gear_r.r[0][p - 1];
          const double cc = r0 * wrms(x);
          if (cc < 1.) { convOK = 1; iterConvergence = newtonK; lab = L_CORR_DONE; break; }
          if (newtonK > 1 && cc > 2. * oldCC) { convOK = 0; iterConvergence = newtonK; lab = L_CORR_DONE; break; }
          oldCC = cc;
          double vn = b * r0 + v[0];
          if (al) {
            if (vn < lo) { vn = lo; b = (lo - z[0]) / r0; }
            if (vn > hi) { vn = hi; b = (hi - z[0]) / r0; }
          }
          va = vn;
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
              fail_keep_z(iterConvergenceFailure >= 50u ? -5 : -6);
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
            double bb = b;
            const double vr = bb * r0;
            double x0 = v[0];
            const double x1 = v[1];
            if (al) {
              if (x0 + vr < lo) { bb = lo - z[0] - x1; x0 = lo - vr; if (x0 < lo) x0 = lo; }
              if (x0 + vr > hi) { bb = hi - z[0] - x1; x0 = hi - vr; if (x0 > hi) x0 = hi; }
            }
            v[0] = x0 + vr;
            v[1] = x1 + bb;
            b = bb;
#pragma unroll
            for (unsigned i = 2; i < 8; ++i)
              if (i <= p) v[i] += b * c_gear_r.r[i][p - 1];
            set8(v, p + 1, (get8(v, p) - get8(z, p)) / (double(p) + 1.));
            if (iterOrder >= p) set8(v, p + 2, (get8(v, p + 1) - get8(z, p + 1)) / (double(p) + 2.));
            dv = true;
          }
          // error test (:876-962)
          double hCur = c_gear_r.Ep[p] * wrms(get8(v, p + 1));
          if (hCur > 1.) {
            iterErrorFailure++;
            ++cerr;
            if (iterErrorFailure >= 50u || fabs(h) <= 0.) {
              fail_keep_z(iterErrorFailure >= 50u ? -4 : -6);
              t = tInMeshPoint;
              lab = L_FINISH;
              break;
            }
            hScaleMax = 1.;
            hCur = 0.8 * pow_ol(1. / hCur, 1. / double(p + 1));
            hScale = hCur;
            if (p > 1u) {
              double hMinus = c_gear_r.Ep[p - 1] * wrms(get8(v, p));
              hMinus = 1. / (hMinus + kMachEpsFloat);
              hMinus = 0.8 * pow_ol(hMinus, 1. / double(p));
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
              load_j();
              const double s = rowdot_ol<double, W>(Js, v[0] - z[0], n, ld, lane, gm);
              const double vr = v[1] - (s * h + z[1]);
              const double normd = wsum_g<W>(gm, al ? fabs(vr) : 0.);
              const double normf = wsum_g<W>(gm, al ? fabs(v[1]) : 0.);
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
              const HCand hc = order_candidates<W>(get8(v, p), get8(v, p + 1), get8(v, p + 2), eps, al, n, gm, p,
                                                   p > 1u && odeOrderStatus != O_INC,
                                                   p < maximum_order && odeOrderStatus != O_DEC,
                                                   alfa2(p - 1), alfa2(p), alfa2(p + 1));
              const double hMinus = hc.hMinus, hC = hc.hC, hPlus = hc.hPlus, alfa1 = hc.alfa1, alfa3 = hc.alfa3;
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
#pragma unroll
          for (unsigned i = 0; i < 8; ++i)
            if (i <= p + 2) z[i] = v[i];
          z[0] = clamp(z[0]);
          dz = true;
          numberOfSteps++;
          ++cstep;
          if (tOut == t) {
            va = z[0];
            lab = L_FINISH;
            break;
          }
          if (tOut < t) {
            // Interpolation (:687-706); the RHS at tOut then sets QR (:599-611)
            const double hp = (tOut - t) / hNordsieck;
            double yv = z[0];
            if (hp != 0.) {
              double hr = 1.;
#pragma unroll
              for (unsigned i = 1; i < 8; ++i) {
                if (i <= p) {
                  hr *= hp;
                  yv += z[i] * hr;
                }
              }
              yv = clamp(yv);
            }
            va = yv;
            phase = PH_FINAL;
            lab = L_NONE;
            break;
          }
          lab = L_START_STEP;
          break;
        }
        case L_FINISH: {
          // utilities.H:153-200 and the scatter of chemistry_DI.H:221-235
          const double s = wsum_g<W>(gm, lane < NC ? va : 0.);
          if (lane < NC) a.Y[(long)lane * a.ld + cell] = va / s;
          if (o.energy && lane == NC) a.T[cell] = va;
          if (lane == 0) {
            if (a.Q) a.Q[cell] = QR;
            if (a.status) a.status[cell] = status;
            if (a.nsteps) a.nsteps[cell] = (int)numberOfSteps;
          }
          phase = PH_DONE;
          lab = L_NONE;
          break;
        }
        default:
          lab = L_NONE;
          break;
      }
    }
    // ---- write the state back ----
    if (al) {
      if (dz)
#pragma unroll
        for (int i = 0; i < 8; ++i) R[RL.oz + i * n + lane] = z[i];
      if (dv)
#pragma unroll
        for (int i = 0; i < 8; ++i) R[RL.ov + i * n + lane] = v[i];
      R[RL.ob + lane] = b;
      R[RL.ova + lane] = va;
      R[RL.ovb + lane] = vb;
      R[RL.oeps + lane] = eps;
    }
    if (lane == 0) {
      R[D_T] = t; R[D_TOUT] = tOut; R[D_TMESH] = tInMeshPoint; R[D_TSTAB] = tStabilize; R[D_H] = h;
      R[D_HNEXT] = hNextStep; R[D_HNORD] = hNordsieck; R[D_HSCALE] = hScale; R[D_HSCALEMAX] = hScaleMax;
      R[D_A24] = alfa2_4; R[D_A25] = alfa2_5; R[D_OLDCC] = oldCC; R[D_HF] = hf; R[D_HJ] = hJ;
      R[D_PENDHS] = pendHScale; R[D_HR0] = hr0f;
      RI[I_PHASE] = phase; RI[I_STATUS] = status; RI[I_P] = (int)p; RI[I_ITORDER] = (int)iterOrder;
      RI[I_ORDNEXT] = (int)orderInNextStep; RI[I_HSTAT] = odeHStatus; RI[I_OSTAT] = odeOrderStatus;
      RI[I_FACTORIZED] = factorized; RI[I_JACCHANGE] = jacobianChange; RI[I_CONVOK] = convOK;
      RI[I_NSTEPS] = (int)numberOfSteps; RI[I_ITCONV] = (int)iterConvergence;
      RI[I_ITCONVRATE] = (int)iterConvergenceRate; RI[I_ITCONVFAIL] = (int)iterConvergenceFailure;
      RI[I_ITERRFAIL] = (int)iterErrorFailure; RI[I_NCFOM] = (int)nConvFailOrderMax;
      RI[I_STEPLASTJ] = (int)stepOfLastJacobian; RI[I_ITCONST] = (int)iterConstSteps;
      RI[I_ITMINORD] = (int)iterMinimumOrder; RI[I_FIXEDMIN] = fixedOrderMin ? 1 : 0;
      RI[I_NEWTONK] = (int)newtonK; RI[I_JCOL] = jcol; RI[I_MAXORD] = (int)maximum_order;
      RI[I_CNT0 + CNT_STEPS] += cstep; RI[I_CNT0 + CNT_JAC] += cjac; RI[I_CNT0 + CNT_FACT] += cfact;
      RI[I_CNT0 + CNT_SOLVE] += csolve; RI[I_CNT0 + CNT_ERRFAIL] += cerr; RI[I_CNT0 + CNT_CONVFAIL] += cconv;
    }
    if (phase == PH_DONE && a.counters) {
      __syncwarp(gm);
      if (lane < NCNT) a.counters[(long)cell * NCNT + lane] = RI[I_CNT0 + lane];
    }
    drain();   // no copy may still be landing in this warp's shared memory when the next cell starts
    __syncwarp(gm);
  }
}


// ---------------------------------------------------------------------------
// Fused lane-group form (LSG_TILE_GROUP): one lane group (16 lanes for up to
// 16 ODE components, else 32) integrates one cell from start to finish.  The
// solver state lives in registers (lane k holds component k of every vector)
// and the group's Jacobian, G^-1 and Gauss-Jordan work arrays in shared
// memory for the cell's whole integration; every RHS the solver asks for is
// evaluated at once by the group (rhs_group), so nothing round-trips through
// HBM between requests.  Cells come from a device queue; the grid is
// persistent.  The solver is the round scheme's state machine, unchanged.
// ---------------------------------------------------------------------------
constexpr int kGW = 4;   // warps per block of the group kernel

// Group-cooperative RHS of the constant-pressure (rho0 == 0) or constant-volume
// reactor (BatchReactorHomogeneousConstantPressure.H:175-223,
// BatchReactorHomogeneousConstantVolume.H:148-199): lane i < NC owns species
// i, lane NC the temperature; reactions are spread over the lanes (C, G, NET:
// the group's shared arrays).  Returns this lane's f; sets QR.
template <int W>
__device__ __noinline__ double rhs_group(const MechLayout* __restrict__ Lp, const double* __restrict__ Md,
                                         const int* __restrict__ Mi, double* __restrict__ C, double* __restrict__ G,
                                         double* __restrict__ NET, double yl, double P0, int energy, double rho0,
                                         int lane, unsigned gm, double* QRout) {
  const MechLayout& L = *Lp;
  const MechView M{Md, Mi};
  const int NC = L.nc, NR = L.nr;
  const double* MW = M.D(L.mw);
  const bool sp = lane < NC;
  const double mwl = sp ? MW[lane] : 1.;
  const double T = __shfl_sync(gm, yl, NC, W);
  const double MWmix = 1. / wsum_g<W>(gm, sp ? yl / mwl : 0.);
  const bool cv = rho0 > 0.;
  const double cTot = cv ? rho0 / MWmix : P0 / kRgas / T;
  const double rho = cv ? rho0 : cTot * MWmix;
  const double Pk = cv ? cTot * kRgas * T : P0;
  const double* TM = M.D(L.t_mid);
  const double T2 = T * T, T3 = T2 * T, T4 = T3 * T, uT = 1. / T;
  const double logT = log(T);
  const double lP = log(101325. / kRgas / T);
  double xl = 0., cl = 0., hrt = 0.;
  if (sp) {
    xl = MWmix * yl;
    xl = xl / mwl;
    cl = cTot * xl;
    C[lane] = cl;
    const bool hiT = T > TM[lane];
    const double* A = hiT ? M.D(L.dh_ht) + 6 * lane : M.D(L.dh_lt) + 6 * lane;
    hrt = A[0] + T * A[1] + T2 * A[2] + T3 * A[3] + T4 * A[4] + uT * A[5];
    const double* B = hiT ? M.D(L.ds_ht) + 6 * lane : M.D(L.ds_lt) + 6 * lane;
    G[lane] = hrt - (B[0] * logT + T * B[1] + T2 * B[2] + T3 * B[3] + T4 * B[4] + B[5]);
  }
  const double cTotSum = wsum_g<W>(gm, cl);
  __syncwarp(gm);
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
  const int* op = M.I(L.ford_ptr);
  const int* osp = M.I(L.ford_sp);
  const double* onu = M.D(L.ford_val);
  const int* pp = M.I(L.prod_ptr);
  const int* psp = M.I(L.prod_sp);
  const double* pnu = M.D(L.prod_nu);
  for (int j = lane; j < NR; j += W) {
    double kArr = exp(lnA[j] + beta[j] * logT - eor[j] * uT);
    if (sgn[j] < 0) kArr *= -1.;
    if (L.n_plog > 0) {
      const int ps = M.I(L.plog_slot)[j];
      if (ps >= 0) kArr = plog_k(M, L, ps, T, logT, Pk);
    }
    if (L.n_cheb > 0) {
      const int cs = M.I(L.cheb_slot)[j];
      if (cs >= 0) kArr = cheb_k(M, L, cs, T, Pk);
    }
    if (L.n_xplog > 0) {
      const int xs = M.I(L.xplog_slot)[j];
      if (xs >= 0) kArr = xplog_k(M, L, xs, T, logT, Pk, cTotSum, [&](int k) { return C[k]; });
    }
    double kMod = kArr;
    const int tb = tbs[j];
    if (tb >= 0) {
      double Mc = cTotSum;
      const int* tp = M.I(L.tb_ptr);
      const int* ts = M.I(L.tb_sp);
      const double* te = M.D(L.tb_eff);
      for (int q = tp[tb]; q < tp[tb + 1]; ++q) Mc += C[ts[q]] * te[q];
      kMod *= Mc;
    }
    const int fo = fos[j];
    if (fo >= 0) {
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
        for (int q = fp[fo]; q < fp[fo + 1]; ++q) Mc += C[fs[q]] * fe[q];
      } else {
        Mc = C[single] + 1.e-16;
      }
      const double Pr = kArr * Mc / kInf;
      const bool cabr = M.I(L.fo_cabr)[fo] != 0;
      double wF = 1.;
      if (ty == 1) {
        double v = (1. - a) * exp(-T / b) + a * exp(-T / c);
        if (d != 0.) v += exp(-d / T);
        const double lF = (v < 1.e-300) ? -300. : log10(v);
        double qq;
        if (Pr > 1.e-32 || cabr) {
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
        wF = pow(lF, 1. / (1. + l10 * l10)) * d;
        const double e = M.D(L.fo_e)[fo];
        if (e != 0.) wF *= pow(T, e);
      }
      if (cabr) kMod *= (1. / (1. + Pr)) * wF;
      else kMod *= kInf * (Pr / (1. + Pr)) * wF / kArr;
    }
    if (L.n_xfo > 0) {
      const int xs = M.I(L.xfo_slot)[j];
      if (xs >= 0) {
        kArr = xfo_k(M, L, xs, T, cTotSum, [&](int k) { return C[k]; });
        kMod = kArr;
      }
    }
    double fwd = 1.;
    for (int q = op[j]; q < op[j + 1]; ++q) fwd *= conc_factor_r(onu[q], C[osp[q]]);
    double net = fwd;
    const int kind = rk[j];
    if (kind != 0) {
      double rv = 1.;
      for (int q = pp[j]; q < pp[j + 1]; ++q) rv *= conc_factor_r(pnu[q], C[psp[q]]);
      double rf;
      if (kind == 1) {
        double dg = 0.;
        for (int q = pp[j]; q < pp[j + 1]; ++q) dg += contrib_r(pnu[q], G[psp[q]]);
        for (int q = rp[j]; q < rp[j + 1]; ++q) dg -= contrib_r(rnu[q], G[rsp[q]]);
        rf = exp(dg - lP * dnu[j]);
      } else {
        const int sr = rs[j];
        rf = exp(M.D(L.rev_lnA)[sr] + M.D(L.rev_beta)[sr] * logT - M.D(L.rev_eor)[sr] * uT) / kArr;
      }
      rv *= rf;
      net -= rv;
    }
    NET[j] = net * kMod;
  }
  __syncwarp(gm);
  double Rl = 0.;
  if (sp) {   // StoichiometricMap::FormationRatesFromReactionRates (:656-729), gathered per species
    const int* fp = M.I(L.fr_ptr);
    const int* fr = M.I(L.fr_rxn);
    const double* fc = M.D(L.fr_coef);
    for (int q = fp[lane]; q < fp[lane + 1]; ++q) {
      const double cf = fc[q];
      Rl += contrib_r(cf < 0. ? -cf : cf, NET[fr[q]]) * (cf < 0. ? -1. : 1.);
    }
  }
  double out = sp ? mwl * Rl / rho : 0.;
  double QR = 0.;
  if (energy) {
    double cpl = 0.;
    if (sp) {
      const bool hiT = T > TM[lane];
      const double* A = hiT ? M.D(L.cp_ht) + 5 * lane : M.D(L.cp_lt) + 5 * lane;
      cpl = (A[0] + T * A[1] + T2 * A[2] + T3 * A[3] + T4 * A[4]) * (cl / cTot);
    }
    const double cpm = kRgas * wsum_g<W>(gm, cpl);
    const double dsum = wsum_g<W>(gm, sp ? Rl * hrt : 0.);
    QR = -dsum * kRgas * T;
    double dT;
    if (cv) {
      const double CvMixMass = (cpm - kRgas) / MWmix;
      const double sumR = wsum_g<W>(gm, sp ? Rl : 0.);
      dT = (QR + kRgas * T * sumR) / (rho0 * CvMixMass);
    } else {
      dT = QR / (rho * (cpm / MWmix));
    }
    if (lane == NC) out = dT;
  }
  __syncwarp(gm);   // C, G, NET may be rewritten by the next call
  *QRout = QR;
  return out;
}

template <typename LUT, int W, int MB>
__global__ void __launch_bounds__(kGW * 32, MB) group_kernel(MechLayout Lp, const unsigned char* __restrict__ mech_gmem,
                                                             StepOptions o, StepArgs a, int* queue, int* err) {
  extern __shared__ __align__(16) unsigned char gsm[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ MechLayout sL;
  if (threadIdx.x == 0) sL = Lp;
  if (!stage_bulk(gsm, mech_gmem, Lp.bytes, &mbar, err)) return;
  const double* Md = (const double*)gsm;
  const int* Mi = (const int*)(gsm + (size_t)Lp.n_double * sizeof(double));
  constexpr int CPW = 32 / W;
  constexpr int GB = kGW * CPW;   // lane groups per block
  const int NC = Lp.nc, NR = Lp.nr;
  const int n = NC + 1, ld = row_ld(n), la = 2 * n + 1;
  const int wl = threadIdx.x & 31;
  const int lane = wl & (W - 1);
  const int w = (threadIdx.x >> 5) * CPW + wl / W;
  const unsigned gm = W == 32 ? kFull : (0xffffu << (wl & 16));
  // per group: C[NC], G[NC], NET[NR], J[n][ld] (double); G^-1 X[n][ld], A[n][2n+1], K[2n] (LUT)
  double* gbase = (double*)(gsm + ((Lp.bytes + 15u) & ~15u));
  const size_t gd = (size_t)2 * NC + NR + (size_t)n * ld;
  double* C = gbase + (size_t)w * gd;
  double* Gs = C + NC;
  double* NET = Gs + NC;
  double* Js = NET + NR;
  LUT* lbase = (LUT*)(gbase + (size_t)GB * gd);
  const size_t gl = (size_t)n * ld + (size_t)n * la + 2 * n;
  LUT* Xs = lbase + (size_t)w * gl;
  LUT* As = Xs + (size_t)n * ld;
  LUT* Ks = As + (size_t)n * la;
  const bool al = lane < n;
  const double lo = lane < NC ? 0. : o.y_min_T, hi = lane < NC ? 1. : o.y_max_T;
  const long max_requests = 4L * (long)o.max_steps * (NC + 10) + 64;
  for (;;) {
    int cell = 0;
    if (lane == 0) cell = atomicAdd(queue, 1);
    cell = __shfl_sync(gm, cell, 0, W);
    if (cell >= a.ncells) break;
    const double rho0 = a.rho ? a.rho[cell] : 0.;
    const double Tc = a.T[cell];
    if (!(Tc > o.tmin_chem)) {   // chemistry_DI.H:92-96: the cell is skipped, its Y renormalised
      const double yv = lane < NC ? a.Y[(long)lane * a.ld + cell] : 0.;
      const double sy = wsum_g<W>(gm, yv);
      if (lane < NC) a.Y[(long)lane * a.ld + cell] = yv / sy;
      if (lane == 0) {
        if (a.status) a.status[cell] = 0;
        if (a.nsteps) a.nsteps[cell] = 0;
      }
      if (a.counters && lane < NCNT) a.counters[(long)cell * NCNT + lane] = 0;
      continue;
    }
    // gather, clip and renormalise (chemistry_DI.H:97-129); solver reset (MultiValueSolver.hpp:367-420)
    double va = 0.;
    if (lane < NC) {
      va = a.Y[(long)lane * a.ld + cell];
      if (va < 0.) va = 0.;
    }
    const double sy = wsum_g<W>(gm, va);
    if (lane < NC) va /= sy;
    if (lane == NC) va = Tc;
    const double t0 = a.t0;
    double t = t0, tOut = t0, tInMeshPoint = t0, tStabilize = t0, h = 0., hNextStep = 0., hNordsieck = 0.;
    double hScale = 0., hScaleMax = 1000., alfa2_4 = o.alfa2_4, alfa2_5 = o.alfa2_5, oldCC = 0., hf = 0., hJ = 0.;
    double pendHScale = 0., hr0f = 0., QR = 0.;
    int status = 1;
    unsigned p = 1, iterOrder = 0, orderInNextStep = 1;
    unsigned maxIterationsJacobian = 20u + 5u * (unsigned)(n - 3);
    if (maxIterationsJacobian > 50u && n < 80) maxIterationsJacobian = 50u;
    int odeHStatus = 1, odeOrderStatus = 1, factorized = 0, jacobianChange = 1, convOK = 1;
    unsigned numberOfSteps = 0, iterConvergence = 0, iterConvergenceRate = 0, iterConvergenceFailure = 0;
    unsigned iterErrorFailure = 0, nConvFailOrderMax = 0, stepOfLastJacobian = 0, iterConstSteps = 0;
    unsigned iterMinimumOrder = 0;
    bool fixedOrderMin = false;
    unsigned newtonK = 0;
    int jcol = 0;
    unsigned maximum_order = (unsigned)o.maximum_order;
    int cstep = 0, csolve = 0, cjac = 0, cfact = 0, cerr = 0, cconv = 0;
    long crhs = 0, cjrhs = 0;
    double z[8], v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) { z[i] = 0.; v[i] = 0.; }
    double b = 0., f = 0., f0 = 0., vb = 0., eps = 0.;
    double x = 0.;
    bool dz = false, dv = false;
    (void)dz; (void)dv; (void)hJ; (void)jcol;
    enum : int { H_DEC = 0, H_CONST = 1, H_INC = 2 };
    enum : int { O_DEC = 0, O_CONST = 1, O_INC = 2 };
    auto alfa2 = [&](unsigned k) { return k == 4 ? alfa2_4 : (k == 5 ? alfa2_5 : .8); };
    auto wrms = [&](double xv) { return wrms_ol<W>(xv, eps, al, n, gm); };
    auto clamp = [&](double y) {
      if (al) {
        if (y < lo) y = lo;
        if (y > hi) y = hi;
      }
      return y;
    };
    auto load_j = [&]() {};   // the Jacobian stays in the group's shared memory
    auto solve = [&](double rhs) {
      const bool fp32 = sizeof(LUT) == sizeof(float);
      ++csolve;
      return solve_ol<LUT, W>(Xs, Js, rhs, hr0f, n, lane, gm, fp32 ? kRefineR : 0);
    };
    auto factorize = [&]() {
      gj_inverse<LUT, W>(Js, As, Ks, Xs, (LUT*)nullptr, hr0f, n, lane, gm);
      ++cfact;
    };
    auto fail_keep_z = [&](int st) {
      status = st;
      va = z[0];
    };
    auto rhs = [&](double yv) {
      ++crhs;
      return rhs_group<W>(&sL, Md, Mi, C, Gs, NET, yv, a.p, o.energy, rho0, lane, gm, &QR);
    };
    auto write_counters = [&]() {
      if (a.counters && lane == 0) {
        long long* cc = a.counters + (long)cell * NCNT;
        cc[CNT_STEPS] = cstep; cc[CNT_RHS] = crhs; cc[CNT_JAC] = cjac; cc[CNT_FACT] = cfact;
        cc[CNT_SOLVE] = csolve; cc[CNT_ERRFAIL] = cerr; cc[CNT_CONVFAIL] = cconv; cc[CNT_JAC_RHS] = cjrhs;
      }
    };
    int phase = PH_INIT;
    f = rhs(va);
    for (long req = 0; phase != PH_DONE; ++req) {
      if (req > 0) {
        // serve the request the solver ended on
        if (req > max_requests) {   // the round scheme's round limit: status -1, last accepted state
          status = -1;
          va = z[0];
          const double sv = wsum_g<W>(gm, lane < NC ? va : 0.);
          if (lane < NC) a.Y[(long)lane * a.ld + cell] = va / sv;
          if (o.energy && lane == NC) a.T[cell] = va;
          if (lane == 0) {
            if (a.Q) a.Q[cell] = QR;
            if (a.status) a.status[cell] = status;
            if (a.nsteps) a.nsteps[cell] = (int)numberOfSteps;
          }
          write_counters();
          break;
        }
        if (phase == PH_PRED) {
          f0 = rhs(vb);
        } else if (phase == PH_JAC) {
          // KernelDense::NumericalJacobian, constrained branch (KernelDense.hpp:111-193): column j by the group
          for (int j = 0; j < n; ++j) {
            double hj = 0.;
            if (lane == j) {
              const double aa = fabs(vb), bb2 = fabs(1. / eps);
              hj = sqrt(kMachEpsDouble) * (aa > bb2 ? aa : bb2);
              hj = fmax(hj, hf / eps);
              hj = fmax(hj, sqrt(kTinyFloat));
              if (vb + hj > (j < n - 1 ? 1. : o.y_max_T)) hj = -hj;
            }
            hj = __shfl_sync(gm, hj, j, W);
            const double fj = rhs_group<W>(&sL, Md, Mi, C, Gs, NET, lane == j ? vb + hj : vb, a.p, o.energy, rho0,
                                           lane, gm, &QR);
            if (al) Js[lane * ld + j] = (1. / hj) * (fj - f0);
            if (j == n - 1) f = fj;
          }
          __syncwarp(gm);
          cjrhs += n;
        } else if (phase == PH_STAB_CONV || phase == PH_STAB_ERR) {
          f = rhs(z[0]);
        } else {   // PH_NEWTON, PH_FINAL
          f = rhs(va);
        }
      }
        enum : int { L_NONE, L_START_STEP, L_DRIVER_LOOP, L_JAC_COLUMN, L_AFTER_JAC, L_AFTER_FACT, L_NEWTON_TEST,
                     L_CORR_DONE, L_FINISH };
        int lab = L_NONE;
        switch (phase) {
          case PH_INIT: {
            // MultiValueSolver::Solve, first call (:445-469)
            const bool illegal = al && (va < lo || va > hi);
            if (__any_sync(gm, illegal)) { status = -9; lab = L_FINISH; break; }
            eps = al ? 1. / (o.atol + o.rtol * fabs(va)) : 0.;
            double lo0, hi0;
            if (t0 != 0.) { lo0 = 100. * kMachEpsDouble * fabs(t0); hi0 = fabs(t0); }
            else { lo0 = kMachEpsDouble; hi0 = 1.e-4; }
            double h0 = 0.5 / (wrms(f) + kMachEpsFloat);
            if (h0 < lo0) h0 = lo0;
            if (h0 > hi0) h0 = hi0;
            const double dtc = a.dt ? a.dt[cell] : a.dt_scalar;
            tOut = t0 + dtc;
            h0 *= fabs(tOut - t0) / (tOut - t0);
            z[0] = va;
            z[1] = f * h0;
            dz = true;
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
              hf = 1.e+3 * kMachEpsDouble * fabs(h) * wrms(f0) * double(n);
              if (hf < 1.e-10) hf = 1.;
              jcol = 0;
              lab = L_JAC_COLUMN;
              break;
            }
            lab = L_AFTER_JAC;
            break;
          }
          case PH_JAC: {
            // the RHS kernel has built every column of J
            ++cjac;
            factorized = 0;
            lab = L_AFTER_JAC;
            break;
          }
          case PH_NEWTON: {
            x = solve(al ? f * h - v[1] - b : 0.);
            b += x;
            ++newtonK;
            if (newtonK > 4u) { convOK = 0; iterConvergence = 4; lab = L_CORR_DONE; }
            else lab = L_NEWTON_TEST;
            break;
          }
          case PH_STAB_CONV: {
            z[1] = f * h;
            dz = true;
            tStabilize = tInMeshPoint;
            if (numberOfSteps > stepOfLastJacobian + 5u) jacobianChange = 1;
            if (numberOfSteps != stepOfLastJacobian && iterConvergenceFailure == 50u) jacobianChange = 1;
            hNextStep *= pendHScale;
            lab = L_DRIVER_LOOP;
            break;
          }
          case PH_STAB_ERR: {
            z[1] = f * h;
            dz = true;
            tStabilize = tInMeshPoint;
            odeHStatus = H_DEC;
            hNextStep *= hScale;
            lab = L_DRIVER_LOOP;
            break;
          }
          default:   // PH_FINAL
            lab = L_FINISH;
            break;
        }

        // labels that need no RHS; a request or a finish is reached within a few hops
        for (int hop = 0; lab != L_NONE; ++hop) {
          if (hop >= 64) {
            fail_keep_z(-10);
            lab = L_FINISH;
          }
          switch (lab) {
            case L_START_STEP: {
              // MultiValueSolver::Solve loop (:532-560) + DriverStep prologue (:753-776)
              if (numberOfSteps >= (unsigned)o.max_steps) { fail_keep_z(-1); lab = L_FINISH; break; }
              eps = al ? 1. / (o.atol + o.rtol * fabs(z[0])) : 0.;
              if (kMachEpsDouble * wrms(z[0]) > 1.) { fail_keep_z(-2); lab = L_FINISH; break; }
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
                double hr = 1.;
    #pragma unroll
                for (unsigned i = 1; i < 8; ++i) {
                  if (i <= p) {
                    hr *= hScale;
                    z[i] *= hr;
                  }
                }
                z[0] = clamp(z[0]);
                dz = true;
                iterOrder = 0;
                odeHStatus = H_CONST;
              }
              h = hNextStep;
              hNordsieck = hNextStep;
              t = tInMeshPoint + h;
              if (t == tInMeshPoint) {
                fail_keep_z(-6);
                t = tInMeshPoint;
                lab = L_FINISH;
                break;
              }
              {
                // MultiValueStep prediction v = D z with min/max handling, then vb = CheckConstraints(v0)
                double wv[8];
    #pragma unroll
                for (int i = 0; i < 8; ++i) wv[i] = (i <= (int)p) ? z[i] : 0.;
    #pragma unroll
                for (int i = 0; i < 7; ++i)
    #pragma unroll
                  for (int j = 6; j >= 0; --j)
                    if (i < (int)p && j >= i && j <= (int)p - 1) wv[j] += wv[j + 1];
                if (al) {
                  if (wv[0] < lo && fabs(wv[0] - lo) * eps < double(n)) {
                    wv[1] = lo - z[0];
                    wv[0] = lo;
    #pragma unroll
                    for (int i = 2; i < 8; ++i) wv[i] = 0.;
                  }
                  if (wv[0] > hi && fabs(wv[0] - hi) * eps < double(n)) {
                    wv[1] = hi - z[0];
                    wv[0] = hi;
    #pragma unroll
                    for (int i = 2; i < 8; ++i) wv[i] = 0.;
                  }
                }
    #pragma unroll
                for (int i = 0; i < 8; ++i)
                  if (i <= (int)p) v[i] = wv[i];
                dv = true;
                vb = clamp(wv[0]);
              }
              phase = PH_PRED;
              lab = L_NONE;
              break;
            }
            case L_JAC_COLUMN: {
              // KernelDense::NumericalJacobian: the RHS kernel evaluates all n perturbed states next
              phase = PH_JAC;
              lab = L_NONE;
              break;
            }
            case L_AFTER_JAC: {
              if (factorized && iterOrder == 0) factorized = 0;
              if (!factorized) {
                hr0f = h * c_gear_r.r[0][p - 1];
                factorize();
                factorized = 1;
              }
              lab = L_AFTER_FACT;
              break;
            }
            case L_AFTER_FACT: {
              x = solve(al ? f0 * h - v[1] : 0.);
              b = x;
              newtonK = 1;
              lab = L_NEWTON_TEST;
              break;
            }
            case L_NEWTON_TEST: {
              const double r0 = c_gear_r.r[0][p - 1];
              const double cc = r0 * wrms(x);
              if (cc < 1.) { convOK = 1; iterConvergence = newtonK; lab = L_CORR_DONE; break; }
              if (newtonK > 1 && cc > 2. * oldCC) { convOK = 0; iterConvergence = newtonK; lab = L_CORR_DONE; break; }
              oldCC = cc;
              double vn = b * r0 + v[0];
              if (al) {
                if (vn < lo) { vn = lo; b = (lo - z[0]) / r0; }
                if (vn > hi) { vn = hi; b = (hi - z[0]) / r0; }
              }
              va = vn;
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
                  fail_keep_z(iterConvergenceFailure >= 50u ? -5 : -6);
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
                double bb = b;
                const double vr = bb * r0;
                double x0 = v[0];
                const double x1 = v[1];
                if (al) {
                  if (x0 + vr < lo) { bb = lo - z[0] - x1; x0 = lo - vr; if (x0 < lo) x0 = lo; }
                  if (x0 + vr > hi) { bb = hi - z[0] - x1; x0 = hi - vr; if (x0 > hi) x0 = hi; }
                }
                v[0] = x0 + vr;
                v[1] = x1 + bb;
                b = bb;
    #pragma unroll
                for (unsigned i = 2; i < 8; ++i)
                  if (i <= p) v[i] += b * c_gear_r.r[i][p - 1];
                set8(v, p + 1, (get8(v, p) - get8(z, p)) / (double(p) + 1.));
                if (iterOrder >= p) set8(v, p + 2, (get8(v, p + 1) - get8(z, p + 1)) / (double(p) + 2.));
                dv = true;
              }
              // error test (:876-962)
              double hCur = c_gear_r.Ep[p] * wrms(get8(v, p + 1));
              if (hCur > 1.) {
                iterErrorFailure++;
                ++cerr;
                if (iterErrorFailure >= 50u || fabs(h) <= 0.) {
                  fail_keep_z(iterErrorFailure >= 50u ? -4 : -6);
                  t = tInMeshPoint;
                  lab = L_FINISH;
                  break;
                }
                hScaleMax = 1.;
                hCur = 0.8 * pow_ol(1. / hCur, 1. / double(p + 1));
                hScale = hCur;
                if (p > 1u) {
                  double hMinus = c_gear_r.Ep[p - 1] * wrms(get8(v, p));
                  hMinus = 1. / (hMinus + kMachEpsFloat);
                  hMinus = 0.8 * pow_ol(hMinus, 1. / double(p));
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
                  load_j();
                  const double s = rowdot_ol<double, W>(Js, v[0] - z[0], n, ld, lane, gm);
                  const double vr = v[1] - (s * h + z[1]);
                  const double normd = wsum_g<W>(gm, al ? fabs(vr) : 0.);
                  const double normf = wsum_g<W>(gm, al ? fabs(v[1]) : 0.);
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
                  const HCand hc = order_candidates<W>(get8(v, p), get8(v, p + 1), get8(v, p + 2), eps, al, n, gm, p,
                                                       p > 1u && odeOrderStatus != O_INC,
                                                       p < maximum_order && odeOrderStatus != O_DEC,
                                                       alfa2(p - 1), alfa2(p), alfa2(p + 1));
                  const double hMinus = hc.hMinus, hC = hc.hC, hPlus = hc.hPlus, alfa1 = hc.alfa1, alfa3 = hc.alfa3;
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
    #pragma unroll
              for (unsigned i = 0; i < 8; ++i)
                if (i <= p + 2) z[i] = v[i];
              z[0] = clamp(z[0]);
              dz = true;
              numberOfSteps++;
              ++cstep;
              if (tOut == t) {
                va = z[0];
                lab = L_FINISH;
                break;
              }
              if (tOut < t) {
                // Interpolation (:687-706); the RHS at tOut then sets QR (:599-611)
                const double hp = (tOut - t) / hNordsieck;
                double yv = z[0];
                if (hp != 0.) {
                  double hr = 1.;
    #pragma unroll
                  for (unsigned i = 1; i < 8; ++i) {
                    if (i <= p) {
                      hr *= hp;
                      yv += z[i] * hr;
                    }
                  }
                  yv = clamp(yv);
                }
                va = yv;
                phase = PH_FINAL;
                lab = L_NONE;
                break;
              }
              lab = L_START_STEP;
              break;
            }
            case L_FINISH: {
              // utilities.H:153-200 and the scatter of chemistry_DI.H:221-235
              const double s = wsum_g<W>(gm, lane < NC ? va : 0.);
              if (lane < NC) a.Y[(long)lane * a.ld + cell] = va / s;
              if (o.energy && lane == NC) a.T[cell] = va;
              if (lane == 0) {
                if (a.Q) a.Q[cell] = QR;
                if (a.status) a.status[cell] = status;
                if (a.nsteps) a.nsteps[cell] = (int)numberOfSteps;
              }
              write_counters();
              phase = PH_DONE;
              lab = L_NONE;
              break;
            }
            default:
              lab = L_NONE;
              break;
          }
        }
    }
    __syncwarp(gm);
  }
}

size_t group_smem_bytes(const MechLayout& L, bool lu64, int width) {
  const size_t n = L.nc + 1, ld = (size_t)row_ld((int)n), la = 2 * n + 1;
  const size_t groups = (size_t)kGW * (width == 16 ? 2 : 1);
  const size_t gd = 2 * (size_t)L.nc + L.nr + n * ld;
  const size_t gl = n * ld + n * la + 2 * n;
  return ((L.bytes + 15u) & ~15u) + groups * gd * sizeof(double) + groups * gl * (lu64 ? 8 : 4) + 16;
}

template <typename LUT, int W, int MB>
cudaError_t group_launch(const MechLayout& L, const unsigned char* mech_gmem, const StepOptions& o,
                         const StepArgs& a, int* queue, int* err, int sm_count, cudaStream_t stream) {
  const size_t smem = group_smem_bytes(L, sizeof(LUT) == 8, W);
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  cudaError_t e =
      cudaFuncSetAttribute(group_kernel<LUT, W, MB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int bps = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, group_kernel<LUT, W, MB>, kGW * 32, smem);
  if (e != cudaSuccess) return e;
  if (bps <= 0) return cudaErrorInvalidConfiguration;
  constexpr int GB = kGW * (32 / W);
  const long want = (a.ncells + GB - 1) / GB, cap = (long)sm_count * bps;
  e = cudaMemsetAsync(queue, 0, sizeof(int), stream);
  if (e != cudaSuccess) return e;
  group_kernel<LUT, W, MB><<<(unsigned)(want < cap ? want : cap), kGW * 32, smem, stream>>>(L, mech_gmem, o, a, queue,
                                                                                              err);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// compact: the cells still integrating form the next list, binned by the solver
// path their next advance will take -- Jacobians; predictor results that
// start a Jacobian, that need a factorisation, that need neither; Newton
// iterates; the rest -- so that the cells that share a warp mostly take the
// same path.  Two kernels: count (bin of every entry, per-bin totals) and
// scatter (warp-aggregated appends into each bin's range).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int cell_bin(const RoundBufs& B, int cell) {
  const int* RI = (const int*)(B.rec + (long)cell * B.L.RS + ND_);
  const int ph = RI[I_PHASE];
  if (ph == PH_DONE) return 0;
  if (ph == PH_JAC) return 1;
  if (ph == PH_PRED) {
    // the tests of MethodGear::FindCorrection (MethodGear.hpp:205-240) that the advance makes next
    const bool jac = RI[I_JACCHANGE] != 0 ||
                     (unsigned)RI[I_NSTEPS] >= (unsigned)RI[I_STEPLASTJ] + (unsigned)RI[I_MAXITJ];
    const bool fact = RI[I_FACTORIZED] == 0 || RI[I_ITORDER] == 0;
    return jac ? 2 : (fact ? 3 : 4);
  }
  return ph == PH_NEWTON ? 5 : 6;
}

__global__ void __launch_bounds__(kCT) rounds_count_kernel(RoundBufs B, int par) {
  const int nact = B.nact[par];
  const int* in = par ? B.act1 : B.act0;
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * kCT + threadIdx.x) >> 5;
  const int nw = gridDim.x * (kCT / 32);
  for (int base = gw * 32; base < nact; base += nw * 32) {
    const int idx = base + lane;
    const int bin = idx < nact ? cell_bin(B, in[idx]) : 0;
    if (idx < nact) B.bin[idx] = (unsigned char)bin;
    const unsigned peers = __match_any_sync(kFull, bin);
    if (bin > 0 && lane == __ffs(peers) - 1) atomicAdd(B.bcnt + bin, __popc(peers));
  }
}

__global__ void __launch_bounds__(kCT) rounds_scatter_kernel(RoundBufs B, int par) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *B.rq = 0;   // the next round's RHS kernel takes work from zero
  const int nact = B.nact[par];
  const int* in = par ? B.act1 : B.act0;
  int* out = par ? B.act0 : B.act1;
  int start[kBins + 1];
  start[0] = 0;
  start[1] = 0;
  for (int b = 2; b <= kBins; ++b) start[b] = start[b - 1] + B.bcnt[b - 1];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    B.nact[par ^ 1] = start[kBins] + B.bcnt[kBins];
    B.njac[par ^ 1] = B.bcnt[1];
  }
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * kCT + threadIdx.x) >> 5;
  const int nw = gridDim.x * (kCT / 32);
  for (int base = gw * 32; base < nact; base += nw * 32) {
    const int idx = base + lane;
    const int bin = idx < nact ? B.bin[idx] : 0;
    const unsigned peers = __match_any_sync(kFull, bin);
    const int leader = __ffs(peers) - 1;
    int off = 0;
    if (bin > 0 && lane == leader) off = atomicAdd(B.bcur + bin, __popc(peers));
    off = __shfl_sync(kFull, off, leader);
    if (bin > 0) out[start[bin] + off + __popc(peers & ((1u << lane) - 1u))] = in[idx];
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

size_t list_bytes(long cap) { return ((sizeof(int) * (size_t)cap) + 255) & ~(size_t)255; }

RoundBufs carve(const MechLayout& L, void* base, long cap, bool lu64) {
  RoundBufs B{};
  B.L = rec_layout(L.nc + 1, lu64);
  char* p = (char*)base;
  B.rec = (double*)p;
  p += sizeof(double) * (size_t)B.L.RS * cap;
  B.act0 = (int*)p; p += list_bytes(cap);
  B.act1 = (int*)p; p += list_bytes(cap);
  B.bin = (unsigned char*)p; p += (cap + 255) & ~255L;
  B.nact = (int*)p;
  B.bcnt = B.nact + 4;
  B.bcur = B.bcnt + 8;
  B.rq = B.bcur + 8;
  B.njac = B.nact + 2;
  return B;
}

size_t advance_smem(const MechLayout& L, bool lu64, int w) {
  const size_t n = L.nc + 1;
  const size_t groups = (size_t)kWA * (w == 16 ? 2 : 1);
  const size_t lut = lu64 ? sizeof(double) : sizeof(float);
  return ((groups * (n * (n + 1) + n * (2 * n + 1) + 2 * n) * lut + 7) & ~(size_t)7) + groups * n * (n + 1) * sizeof(double);
}

template <typename LUT, int NM>
cudaError_t prepare_advance(size_t as, int* bps) {
  cudaError_t e = cudaFuncSetAttribute(rounds_advance_kernel<LUT, NM>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)as);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, rounds_advance_kernel<LUT, NM>, kWA * 32, as);
}

}  // namespace

size_t rounds_bytes(const MechLayout& L, long cap, bool lu64) {
  const RecLayout R = rec_layout(L.nc + 1, lu64);
  return sizeof(double) * (size_t)R.RS * cap + 2 * list_bytes(cap) + ((cap + 255) & ~255L) + 256;
}

cudaError_t launch_steady_sources(const MechLayout& L, const unsigned char* mech_gmem, long ncells, const double* Y,
                                  const double* T, long ld, const double* p, double p_scalar, double* scratch,
                                  double* Simp, double* Sexp, long lds, int sm_count, int* err, cudaStream_t stream) {
  if (ncells <= 0) return cudaSuccess;
  const size_t smem = ((L.bytes + 15u) & ~15u) + (size_t)3 * L.nc * kRT * sizeof(double);
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(steady_sources_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int bps = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, steady_sources_kernel, kRT, smem);
  if (e != cudaSuccess) return e;
  if (bps <= 0) return cudaErrorInvalidConfiguration;
  const long want = (ncells + kRT - 1) / kRT, cap = (long)sm_count * bps;
  const long n = L.nc + 1;
  double* yb = scratch;
  double* s0 = scratch + n * ncells;
  double* sp = scratch + 2 * n * ncells;
  steady_sources_kernel<<<(unsigned)(want < cap ? want : cap), kRT, smem, stream>>>(
      L, mech_gmem, ncells, Y, T, ld, p, p_scalar, yb, s0, sp, Simp, Sexp, lds, err);
  return cudaGetLastError();
}

// Jacobians of the constant-pressure reactor for ncells states (lsg_jacobian_device), one thread per
// state: the species columns analytic (analytic_jacobian_species), the temperature column a forward
// difference with the increment hT = sqrt(eps) max(T, 1).  y: species-major [n][ld]; J: [ncells][n][n]
// row-major.
__global__ void __launch_bounds__(kRT) jacobian_kernel(MechLayout Lp, const unsigned char* __restrict__ mech_gmem,
                                                       long ncells, const double* __restrict__ y, long ld, double P0,
                                                       int energy, double* __restrict__ J, int* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ MechLayout sL;
  if (threadIdx.x == 0) sL = Lp;
  if (!stage_bulk(smem, mech_gmem, Lp.bytes, &mbar, err)) return;
  const double* Md = (const double*)smem;
  const int* Mi = (const int*)(smem + (size_t)Lp.n_double * sizeof(double));
  double* scratch = (double*)(smem + ((Lp.bytes + 15u) & ~15u));
  const int n = Lp.nc + 1;
  for (long cell = (long)blockIdx.x * kRT + threadIdx.x; cell < ncells; cell += (long)gridDim.x * kRT) {
    double* Jc = J + cell * (long)n * n;
    analytic_jacobian_species(&sL, Md, Mi, scratch, y + cell, ld, P0, energy, Jc);
    // temperature column: (f(y + hT e_T) - f(y)) / hT; f(y) is parked in the column first
    const double T = y[(long)(n - 1) * ld + cell];
    const double hT = sqrt(kMachEpsDouble) * fmax(fabs(T), 1.);
    rhs_cell(&sL, Md, Mi, scratch, y + cell, ld, -1, 0., Jc + (n - 1), n, P0, energy, 0.);
    double f1[32];
    rhs_cell(&sL, Md, Mi, scratch, y + cell, ld, n - 1, T + hT, f1, 1, P0, energy, 0.);
    for (int i = 0; i < n; ++i) Jc[i * n + n - 1] = (f1[i] - Jc[i * n + n - 1]) / hT;
  }
}

cudaError_t launch_jacobian(const MechLayout& L, const unsigned char* mech_gmem, long ncells, const double* y, long ld,
                            double p, int energy, double* J, int sm_count, int* err, cudaStream_t stream) {
  if (ncells <= 0) return cudaSuccess;
  if (L.nc + 1 > 32) return cudaErrorInvalidValue;
  const size_t smem = ((L.bytes + 15u) & ~15u) + (size_t)3 * L.nc * kRT * sizeof(double);
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(jacobian_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const long want = (ncells + kRT - 1) / kRT, cap = (long)sm_count * 4;
  jacobian_kernel<<<(unsigned)(want < cap ? want : cap), kRT, smem, stream>>>(L, mech_gmem, ncells, y, ld, p, energy,
                                                                             J, err);
  return cudaGetLastError();
}

cudaError_t launch_steady_sources_sparse(const MechLayout& L, const unsigned char* mech_gmem, long ncells,
                                         const double* Y, const double* T, long ld, const double* p, double p_scalar,
                                         int species, int energy, double* scratch, double* Simp, double* Sexp,
                                         long lds, int sm_count, int* err, cudaStream_t stream) {
  if (ncells <= 0) return cudaSuccess;
  const size_t smem = ((L.bytes + 15u) & ~15u) + (size_t)3 * L.nc * kRT * sizeof(double);
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  cudaError_t e =
      cudaFuncSetAttribute(steady_sources_sparse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int bps = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, steady_sources_sparse_kernel, kRT, smem);
  if (e != cudaSuccess) return e;
  if (bps <= 0) return cudaErrorInvalidConfiguration;
  const long want = (ncells + kRT - 1) / kRT, cap = (long)sm_count * bps;
  const long n = L.nc + 1;
  steady_sources_sparse_kernel<<<(unsigned)(want < cap ? want : cap), kRT, smem, stream>>>(
      L, mech_gmem, ncells, Y, T, ld, p, p_scalar, species, energy, scratch, scratch + n * ncells,
      scratch + 2 * n * ncells, Simp, Sexp, lds, err);
  return cudaGetLastError();
}

size_t rounds_cache_bytes(const MechLayout& L, const RoundsPlan& P) {
  return sizeof(double) * (size_t)(L.nc + 1) * (size_t)P.g_rhs * kRT;
}

cudaError_t upload_gear_rounds(const GearConsts& gc) { return cudaMemcpyToSymbol(c_gear_r, &gc, sizeof(GearConsts)); }

cudaError_t rounds_prepare(const MechLayout& L, bool lu64, int sm_count, int width, RoundsPlan* P) {
  const int n = L.nc + 1;
  if (n > 32) return cudaErrorInvalidValue;
  if (width == 0) width = n <= 16 ? 16 : 32;   // default: two cells per warp when they fit
  if ((width != 16 && width != 32) || n > width) return cudaErrorInvalidValue;
  *P = RoundsPlan{};
  P->lu64 = lu64;
  P->w = width;
  P->rhs_smem = ((L.bytes + 15u) & ~15u) + (size_t)3 * L.nc * kRT * sizeof(double);
  P->adv_smem = advance_smem(L, lu64, width);
  cudaError_t e = cudaFuncSetAttribute(rounds_rhs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)P->rhs_smem);
  if (e != cudaSuccess) return e;
  int rhs_bps = 0, adv_bps = 0, cmp_bps = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&rhs_bps, rounds_rhs_kernel, kRT, P->rhs_smem);
  if (e != cudaSuccess) return e;
  if (lu64) e = width == 16 ? prepare_advance<double, 16>(P->adv_smem, &adv_bps) : prepare_advance<double, 32>(P->adv_smem, &adv_bps);
  else e = width == 16 ? prepare_advance<float, 16>(P->adv_smem, &adv_bps) : prepare_advance<float, 32>(P->adv_smem, &adv_bps);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cmp_bps, rounds_scatter_kernel, kCT, 0);
  if (e != cudaSuccess) return e;
  if (rhs_bps <= 0 || adv_bps <= 0 || cmp_bps <= 0) return cudaErrorInvalidConfiguration;
  // persistent grids: every kernel fills the GPU once and strides over the list
  P->g_rhs = (unsigned)(sm_count * rhs_bps);
  P->g_adv = (unsigned)(sm_count * adv_bps);
  P->g_cmp = (unsigned)(sm_count * cmp_bps);
  P->g_init = (unsigned)(sm_count * 8);
  return cudaSuccess;
}

cudaError_t launch_rounds(const RoundsPlan& P, const MechLayout& L, const unsigned char* mech_gmem,
                          const StepOptions& o, const StepArgs& a, void* state, long cap, int* nact_host,
                          long max_rounds, int* err, cudaStream_t stream, long long* launches,
                          KernelTimer* kt) {
  // nact_host: two pinned ints (list length, error flags); launches: kernels enqueued (added to)
  const int n = L.nc + 1;
  if (n > 32 || a.ncells > cap || a.ncells <= 0) return cudaErrorInvalidValue;
  RoundBufs B = carve(L, state, cap, P.lu64);
  B.fsc = (double*)((char*)state + rounds_bytes(L, cap, P.lu64));   // rounds_cache_bytes(L, P) after the rest
  B.rho = a.rho;
  kt->begin(KT_INIT, stream);
  rounds_init_kernel<<<P.g_init, kAT, 0, stream>>>(L.nc, o, a, B);
  kt->end(stream);
  *launches += 1;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int kBatch = 8;   // rounds between host checks of the list length
  int par = 0;
  for (long round = 0; round < max_rounds; round += kBatch) {
    for (int r = 0; r < kBatch; ++r) {
      kt->begin(KT_RHS, stream);
      // the analytic Jacobian is for the constant-pressure reactor without the concentration-dependent
      // extended PLOG / fall-off constants; the other cases keep the differences
      rounds_rhs_kernel<<<P.g_rhs, kRT, P.rhs_smem, stream>>>(L, mech_gmem, o.energy, a.p, o.y_max_T, B, par,
                                                              (o.jacobian != 0 && !a.rho && L.n_xplog == 0 && L.n_xfo == 0) ? 1 : 0,
                                                              err);
      kt->end(stream);
      const dim3 ga(P.g_adv), ta(kWA * 32);
      kt->begin(KT_ADVANCE, stream);
      if (P.lu64) {
        if (P.w == 16) rounds_advance_kernel<double, 16><<<ga, ta, P.adv_smem, stream>>>(L.nc, o, a, B, par);
        else rounds_advance_kernel<double, 32><<<ga, ta, P.adv_smem, stream>>>(L.nc, o, a, B, par);
      } else {
        if (P.w == 16) rounds_advance_kernel<float, 16><<<ga, ta, P.adv_smem, stream>>>(L.nc, o, a, B, par);
        else rounds_advance_kernel<float, 32><<<ga, ta, P.adv_smem, stream>>>(L.nc, o, a, B, par);
      }
      kt->end(stream);
      kt->begin(KT_COMPACT, stream);
      rounds_count_kernel<<<P.g_cmp, kCT, 0, stream>>>(B, par);
      rounds_scatter_kernel<<<P.g_cmp, kCT, 0, stream>>>(B, par);
      kt->end(stream);
      *launches += 4;
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
    kt->collect();
    if (nact_host[0] == 0) return cudaSuccess;
    if (nact_host[1] != 0) return cudaErrorLaunchTimeout;   // a kernel raised a flag: stop, the caller reports it
  }
  return cudaErrorLaunchTimeout;
}


// occupancy: 4 (up to 128 registers a thread) or 2 blocks per SM (up to 255)
template <int MB>
cudaError_t launch_group_mb(const MechLayout& L, const unsigned char* mech_gmem, const StepOptions& o,
                            const StepArgs& a, bool lu64, int* queue, int* err, int sm_count, cudaStream_t stream) {
  if (L.nc + 1 <= 16)
    return lu64 ? group_launch<double, 16, MB>(L, mech_gmem, o, a, queue, err, sm_count, stream)
                : group_launch<float, 16, MB>(L, mech_gmem, o, a, queue, err, sm_count, stream);
  return lu64 ? group_launch<double, 32, MB>(L, mech_gmem, o, a, queue, err, sm_count, stream)
              : group_launch<float, 32, MB>(L, mech_gmem, o, a, queue, err, sm_count, stream);
}

cudaError_t launch_group(const MechLayout& L, const unsigned char* mech_gmem, const StepOptions& o, const StepArgs& a,
                         bool lu64, int min_blocks, int* queue, int* err, int sm_count, cudaStream_t stream) {
  if (a.ncells <= 0) return cudaSuccess;
  if (L.nc + 1 > 32) return cudaErrorInvalidValue;
  return min_blocks == 2 ? launch_group_mb<2>(L, mech_gmem, o, a, lu64, queue, err, sm_count, stream)
                         : launch_group_mb<4>(L, mech_gmem, o, a, lu64, queue, err, sm_count, stream);
}

}  // namespace lsg
