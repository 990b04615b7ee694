// Batched reaction step: one CUDA thread per cell ("lane per cell"),
// persistent grid, device work queue.  Same method as the plain step -- the
// Gear/BDF multivalue solver of math/native-ode-solvers/MultiValueSolver.hpp:423-1328
// with MethodGear.hpp:195-516 and the finite-difference Jacobian of
// KernelDense.hpp:111-193 -- organised for throughput:
//
// * every thread integrates its own cell.  The solver is a state machine that
//   stops at each right-hand-side request, so one loop iteration is "all lanes
//   evaluate one RHS together, then each lane advances its own solver to its
//   next request".  A lane building a finite-difference Jacobian spends its
//   RHS evaluations on its columns while its neighbours spend theirs on Newton
//   iterations; nobody waits for a neighbour's Jacobian;
// * LU factorisations are done warp-cooperatively (lanes = rows) for every
//   lane that needs one, instead of serially on one lane while 31 idle;
// * the mechanism tables are staged once per block into shared memory and are
//   read as warp-wide broadcasts (all lanes walk the same reaction together);
// * per-cell vectors (Nordsieck arrays, Newton vectors, the FP64 Jacobian)
//   live in a slot-interleaved HBM buffer ([element][slot], coalesced); every
//   loop over them goes through helpers with non-aliasing pointers so the
//   loads of a loop are in flight together.  LU factors, pivots, the Newton
//   correction and the RHS scratch live in shared memory;
// * cells are taken from a queue (optionally ordered by measured step counts);
// * LU in FP32 (mixed precision) or FP64.  Rates, the Newton residual, the
//   error estimate and step-size control stay FP64; the Newton iteration
//   refines the FP32 solves against the FP64 residual.
//
// The RHS computes each reaction's rate constants inside the rate loop and
// scatters rates into formation rates (reaction order) instead of gathering
// per species; it agrees with the reference to rounding.
#include <mutex>

#include "lsg_common.cuh"
#include "lsg_kernels.h"

namespace lsg {

static __constant__ GearConsts c_gear_b;

namespace {

constexpr int kBT = 64;        // lanes (cells) per block
constexpr int kLS = kBT + 1;   // padded lane stride of the LU block
constexpr int kRefine = 2;     // refinement sweeps of an FP32-factor solve

enum Phase : int {
  PH_FETCH = 0,
  PH_INIT,       // f(y0)
  PH_PRED,       // f(vb), first Newton evaluation
  PH_JAC,        // f(vb + hJ e_j), FD column jcol
  PH_NEWTON,     // f(va), Newton iterate
  PH_STAB_CONV,  // f(z0) during convergence-failure recovery
  PH_STAB_ERR,   // f(z0) after an error-test failure
  PH_FINAL,      // f(y(tOut)) -> QR
  PH_FACT,       // waiting for the warp-cooperative LU factorisation
};

// element offsets of the per-cell vectors inside a slot (units: doubles)
struct SlotLayout {
  int z, v, b, f, f0, va, vb, eps, r, jac, total;
};

__host__ __device__ inline SlotLayout slot_layout(const MechLayout& L) {
  const int n = L.nc + 1;
  SlotLayout s{};
  int o = 0;
  s.z = o; o += 8 * n;
  s.v = o; o += 8 * n;
  s.b = o; o += n;
  s.f = o; o += n;
  s.f0 = o; o += n;
  s.va = o; o += n;
  s.vb = o; o += n;
  s.eps = o; o += n;
  s.r = o; o += n;
  s.jac = o; o += n * n;   // FP64 Jacobian (the FP64 residual of the refinement uses it)
  s.total = o;
  return s;
}

__device__ __forceinline__ double contrib_b(double nu, double v) {
  if (nu == 1.) return v;
  if (nu == 2.) return v + v;
  if (nu == 3.) return v + v + v;
  if (nu == 0.5) return 0.5 * v;
  return nu * v;
}

__device__ __forceinline__ double conc_factor_b(double nu, double c1) {
  if (nu == 1.) return c1;
  if (nu == 2.) return c1 * c1;
  if (nu == 3.) return c1 * c1 * c1;
  if (nu == 0.5) return sqrt(c1);
  return pow(c1, nu);
}

__device__ __forceinline__ double lo_bound(int k, int NC, double yminT) { return k < NC ? 0. : yminT; }
__device__ __forceinline__ double hi_bound(int k, int NC, double ymaxT) { return k < NC ? 1. : ymaxT; }

// ---------------------------------------------------------------------------
// Thread-serial RHS of the constant-pressure reactor
// (BatchReactorHomogeneousConstantPressure.H:175-223).  y: this lane's input
// vector (stride ns) with component pj replaced by pval when pj >= 0; f: output.
// C,H,S,R scratch in shared memory, [species][lane].  Returns QR.  rho0 > 0
// selects the constant-volume reactor of that density
// (BatchReactorHomogeneousConstantVolume.H:148-199).
// ---------------------------------------------------------------------------
__device__ __noinline__ double rhs_lane(const MechLayout* __restrict__ Lp, const double* __restrict__ Md,
                                        const int* __restrict__ Mi, double* __restrict__ scratch,
                                        const double* __restrict__ y, long ns, int pj, double pval,
                                        double* __restrict__ f, double P0, int energy, double rho0) {
  const MechLayout& L = *Lp;
  const MechView M{Md, Mi};
  const int NC = L.nc, NR = L.nr;
  const int tid = threadIdx.x;
  double* C = scratch;
  double* H = scratch + NC * kBT;
  double* Sx = scratch + 2 * NC * kBT;
  double* R = scratch + 3 * NC * kBT;
#define SC_(arr, i) arr[(i) * kBT + tid]
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
    for (int q = op[j]; q < op[j + 1]; ++q) fwd *= conc_factor_b(onu[q], SC_(C, osp[q]));
    double net = fwd;
    const int kind = rk[j];
    if (kind != 0) {
      double rv = 1.;
      for (int q = pp[j]; q < pp[j + 1]; ++q) rv *= conc_factor_b(pnu[q], SC_(C, psp[q]));
      if (kind == 1) {
        // 1/Keq from reaction enthalpy and entropy (StoichiometricMap.hpp:916-1001, KineticsMap_CHEMKIN.hpp:1217-1222)
        double dh = 0., ds = 0.;
        int qa = rp[j], qb = pp[j];
        const int ae = rp[j + 1], be = pp[j + 1];
        while (qa < ae || qb < be) {
          const int sa = qa < ae ? rsp[qa] : (1 << 30);
          const int sb = qb < be ? psp[qb] : (1 << 30);
          if (sa <= sb) {
            dh -= contrib_b(rnu[qa], SC_(H, sa));
            ds -= contrib_b(rnu[qa], SC_(Sx, sa));
            ++qa;
          } else {
            dh += contrib_b(pnu[qb], SC_(H, sb));
            ds += contrib_b(pnu[qb], SC_(Sx, sb));
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
    for (int q = rp[j]; q < rp[j + 1]; ++q) SC_(R, rsp[q]) -= contrib_b(rnu[q], net);
    for (int q = pp[j]; q < pp[j + 1]; ++q) SC_(R, psp[q]) += contrib_b(pnu[q], net);
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
  f[(long)NC * ns] = dT;
#undef SC_
  return QR;
}

// ---------------------------------------------------------------------------
// Per-lane vector helpers.  Pointers address element 0 of a lane's vector;
// element k is at [k * ns].  __restrict__ lets each loop keep all its loads in
// flight at once (the vectors never overlap).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double wrms(const double* __restrict__ x, const double* __restrict__ e, int n, long ns) {
  double s = 0.;
#pragma unroll 4
  for (int k = 0; k < n; ++k) {
    const double c = x[k * ns] * e[k * ns];
    s += c * c;
  }
  return sqrt(s / double(n));
}

__device__ __forceinline__ void set_eps(const double* __restrict__ w, double* __restrict__ e, int n, long ns,
                                        double atol, double rtol) {
#pragma unroll 4
  for (int k = 0; k < n; ++k) e[k * ns] = 1. / (atol + rtol * fabs(w[k * ns]));
}

// DriverStep rescale of z[1..p] and CheckConstraints(z0) (MultiValueSolver.hpp:780-797)
__device__ __forceinline__ void rescale_z(double* __restrict__ z, int n, long ns, unsigned p, double hScale, int NC,
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
    const double lo = lo_bound(k, NC, yminT), hi = hi_bound(k, NC, ymaxT);
    if (z0 < lo) z0 = lo;
    if (z0 > hi) z0 = hi;
    z[k * ns] = z0;
  }
}

// MultiValueStep prediction v = D z with min/max handling (MultiValueSolver.hpp:1214-1262) and
// FindCorrection's vb = CheckConstraints(v0) (MethodGear.hpp:198-202)
__device__ __forceinline__ void predict(const double* __restrict__ z, double* __restrict__ v,
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
    const double lo = lo_bound(k, NC, yminT), hi = hi_bound(k, NC, ymaxT);
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

}  // namespace

// ---------------------------------------------------------------------------
// Batched kernel.  LUT = float (mixed precision) or double.
// ---------------------------------------------------------------------------
template <typename LUT>
__global__ void __launch_bounds__(kBT, 1)
batched_kernel(MechLayout Lp, const unsigned char* __restrict__ mech_gmem, StepOptions o, StepArgs a,
               double* __restrict__ gz, double* __restrict__ gv, double* __restrict__ gb, double* __restrict__ gf,
               double* __restrict__ gf0, double* __restrict__ gva, double* __restrict__ gvb,
               double* __restrict__ geps, double* __restrict__ gr, double* __restrict__ gjac, long ns,
               const int* __restrict__ order, int* __restrict__ queue, int* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ MechLayout sL;
  if (threadIdx.x == 0) sL = Lp;
  if (!stage_bulk(smem, mech_gmem, Lp.bytes, &mbar, err)) return;
  const double* Md = (const double*)smem;
  const int* Mi = (const int*)(smem + (size_t)Lp.n_double * sizeof(double));
  double* scratch = (double*)(smem + ((Lp.bytes + 15u) & ~15u));
  const int NC = Lp.nc, n = NC + 1;
  // per-lane shared blocks: Newton correction DB[n][kBT], LU[n*n][kLS], pivots[n][kBT]
  double* sDB = scratch + (size_t)4 * NC * kBT;
  LUT* sLU = (LUT*)(sDB + (size_t)n * kBT);
  int* sPIV = (int*)(((size_t)(sLU + (size_t)n * n * kLS) + 15) & ~(size_t)15);
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int wbase = tid & ~31;
  const long slot = (long)blockIdx.x * kBT + tid;
  // each array is its own kernel parameter so the compiler knows they never overlap
  double* const pz = gz + slot;
  double* const pv = gv + slot;
  double* const pb = gb + slot;
  double* const pf = gf + slot;
  double* const pf0 = gf0 + slot;
  double* const pva = gva + slot;
  double* const pvb = gvb + slot;
  double* const peps = geps + slot;
  double* const pr = gr + slot;
  double* const pjac = gjac + slot;   // element e at pjac[e * ns]
  auto DB = [&](int k) -> double& { return sDB[k * kBT + tid]; };
  auto LU = [&](int i, int j) -> LUT& { return sLU[(i * n + j) * kLS + tid]; };
  auto PIV = [&](int k) -> int& { return sPIV[k * kBT + tid]; };
  const double yminT = o.y_min_T, ymaxT = o.y_max_T;
  const double P0 = a.p;

  // ---- per-cell solver state (registers) ----
  long cell = -1;
  int phase = PH_FETCH;
  double QR = 0.;
  double t = 0., t0 = 0., tOut = 0., tInMeshPoint = 0., tStabilize = 0.;
  double h = 0., hNextStep = 0., hNordsieck = 0., hScale = 0., hScaleMax = 1000.;
  double alfa2_4 = .8, alfa2_5 = .8;
  unsigned maximum_order = 5, p = 1, iterOrder = 0, orderInNextStep = 1, maxIterationsJacobian = 50;
  int odeHStatus = 1, odeOrderStatus = 1, factorized = 0, jacobianChange = 1, convOK = 1, status = 0;
  unsigned numberOfSteps = 0, iterConvergence = 0, iterConvergenceRate = 0, iterConvergenceFailure = 0;
  unsigned iterErrorFailure = 0, nConvFailOrderMax = 0, stepOfLastJacobian = 0, iterConstSteps = 0,
           iterMinimumOrder = 0;
  bool fixedOrderMin = false;
  unsigned newtonK = 0;
  double oldCC = 0.;
  int jcol = 0;
  double hf = 0., hJ = 0.;
  unsigned cnt[NCNT] = {};
  double pendHScale = 0.;
  double pendHr0 = 0.;
  enum : int { H_DEC = 0, H_CONST = 1, H_INC = 2 };
  enum : int { O_DEC = 0, O_CONST = 1, O_INC = 2 };
  auto alfa2 = [&](unsigned k) { return k == 4 ? alfa2_4 : (k == 5 ? alfa2_5 : .8); };
  auto Zp = [&](unsigned i) { return pz + (long)i * n * ns; };
  auto Vp = [&](unsigned i) { return pv + (long)i * n * ns; };

  // Forward/back substitution with the factors in shared memory, on DB in place.
  auto lu_subst = [&]() {
    for (int k = 0; k < n; ++k) {
      const int pk = PIV(k);
      if (pk != k) {
        const double tmp = DB(k);
        DB(k) = DB(pk);
        DB(pk) = tmp;
      }
    }
    for (int j = 0; j < n; ++j) {
      const double vj = DB(j);
#pragma unroll 4
      for (int i = j + 1; i < n; ++i) DB(i) -= (double)LU(i, j) * vj;
    }
    for (int j = n - 1; j >= 0; --j) {
      const double xj = DB(j) / (double)LU(j, j);
      DB(j) = xj;
#pragma unroll 4
      for (int i = 0; i < j; ++i) DB(i) -= (double)LU(i, j) * xj;
    }
  };
  // DB <- G^-1 DB, G = I - hr0 J the matrix of the last factorisation.  With
  // FP32 factors the solution is refined against the FP64 residual
  // r - G x (G rebuilt in FP64 from the stored Jacobian) until it is the
  // FP64 solve to rounding.
  auto lin_solve = [&]() {
    if (sizeof(LUT) == sizeof(float)) {
#pragma unroll 4
      for (int k = 0; k < n; ++k) pr[k * ns] = DB(k);
      lu_subst();
      for (int it = 0; it < kRefine; ++it) {
        for (int i = 0; i < n; ++i) {
          double s = 0.;
#pragma unroll 4
          for (int j = 0; j < n; ++j) s += pjac[(long)(i * n + j) * ns] * DB(j);
          pf[i * ns] = pr[i * ns] - (DB(i) - pendHr0 * s);
        }
#pragma unroll 4
        for (int k = 0; k < n; ++k) {
          pva[k * ns] = DB(k);
          DB(k) = pf[k * ns];
        }
        lu_subst();
#pragma unroll 4
        for (int k = 0; k < n; ++k) DB(k) += pva[k * ns];
      }
    } else {
      lu_subst();
    }
    ++cnt[CNT_SOLVE];
  };
  // Warp-cooperative LU of lane q's G = I - hr0 J (lanes = rows); partial
  // pivoting on the largest magnitude, first occurrence.  All 32 lanes call it.
  auto coop_factorize = [&](int qlane, double hr0) {
    const int q = wbase + qlane;
    const double* jq = gjac + ((long)blockIdx.x * kBT + q);
    LUT* lq = sLU + q;
    const int i = lane;
    if (i < n)
      for (int j = 0; j < n; ++j) {
        double g = -hr0 * jq[(long)(i * n + j) * ns];
        if (i == j) g += 1.;
        lq[(i * n + j) * kLS] = (LUT)g;
      }
    __syncwarp();
    for (int k = 0; k < n; ++k) {
      LUT v = (i >= k && i < n) ? (LUT)fabs(lq[(i * n + k) * kLS]) : (LUT)-1;
      int r = i;
      for (int off = 16; off > 0; off >>= 1) {
        const LUT ov = __shfl_xor_sync(kFull, v, off);
        const int orr = __shfl_xor_sync(kFull, r, off);
        if (ov > v || (ov == v && orr < r)) { v = ov; r = orr; }
      }
      // one pivot for the whole warp; a NaN column cannot send it outside rows k..n-1
      r = __shfl_sync(kFull, r, 0);
      if (r < k || r >= n) r = k;
      if (lane == 0) sPIV[k * kBT + q] = r;
      if (r != k && i < n) {
        const LUT tmp = lq[(k * n + i) * kLS];
        lq[(k * n + i) * kLS] = lq[(r * n + i) * kLS];
        lq[(r * n + i) * kLS] = tmp;
      }
      __syncwarp();
      const LUT d = lq[(k * n + k) * kLS];
      if (i > k && i < n) {
        LUT l = lq[(i * n + k) * kLS];
        if (d != (LUT)0) l /= d;
        lq[(i * n + k) * kLS] = l;
        for (int j = k + 1; j < n; ++j) lq[(i * n + j) * kLS] -= l * lq[(k * n + j) * kLS];
      }
      __syncwarp();
    }
  };

  bool done = false;
  for (;;) {
    // =================== fetch a cell (skipped cells handled here) ===================
    while (!done && phase == PH_FETCH) {
      const int qi = atomicAdd(queue, 1);
      if (qi >= a.ncells) { done = true; break; }
      cell = order ? (long)order[qi] : (long)qi;
      const double Tc = a.T[cell];
      if (!(Tc > o.tmin_chem)) {
        double s = 0.;
        for (int i = 0; i < NC; ++i) s += a.Y[(long)i * a.ld + cell];
        for (int i = 0; i < NC; ++i) a.Y[(long)i * a.ld + cell] /= s;
        if (a.status) a.status[cell] = 0;
        if (a.nsteps) a.nsteps[cell] = 0;
        if (a.counters)
          for (int k = 0; k < NCNT; ++k) a.counters[(long)cell * NCNT + k] = 0;
        continue;
      }
      // chemistry_DI.H:100-129: gather, clip, renormalise (y0 kept in va)
      double s = 0.;
      for (int i = 0; i < NC; ++i) {
        double yi = a.Y[(long)i * a.ld + cell];
        if (yi < 0.) yi = 0.;
        pva[i * ns] = yi;
        s += yi;
      }
      for (int i = 0; i < NC; ++i) pva[i * ns] /= s;
      pva[NC * ns] = Tc;
      // SetInitialConditions + ResetMethod + Reset
      t0 = a.t0;
      tOut = t = tInMeshPoint = tStabilize = t0;
      p = 1; iterOrder = 0; orderInNextStep = 1;
      maxIterationsJacobian = 20u + 5u * (unsigned)(n - 3);
      if (maxIterationsJacobian > 50u && n < 80) maxIterationsJacobian = 50u;
      odeHStatus = H_CONST; odeOrderStatus = O_CONST; status = 1;
      factorized = 0; jacobianChange = 1; convOK = 1;
      h = 0.; hNextStep = 0.; hScale = 0.;
      numberOfSteps = 0; nConvFailOrderMax = 0;
      iterConvergence = 0; iterConvergenceRate = 0; iterConvergenceFailure = 0; iterErrorFailure = 0;
      stepOfLastJacobian = 0;
      hNordsieck = 0.; hScaleMax = 1000.;
      fixedOrderMin = false; iterConstSteps = 0; iterMinimumOrder = 0;
      alfa2_4 = o.alfa2_4; alfa2_5 = o.alfa2_5; maximum_order = (unsigned)o.maximum_order;
      for (int k = 0; k < NCNT; ++k) cnt[k] = 0;
      phase = PH_INIT;
    }
    if (__all_sync(kFull, done)) break;
    __syncwarp();

    // =================== one RHS evaluation (all working lanes together) ===================
    if (!done) {
      const double* src = pva;
      double* dst = pf;
      int pj = -1;
      double pval = 0.;
      switch (phase) {
        case PH_PRED: src = pvb; dst = pf0; break;
        case PH_JAC: src = pvb; pj = jcol; pval = pvb[jcol * ns] + hJ; break;
        case PH_STAB_CONV:
        case PH_STAB_ERR: src = pz; break;
        default: break;   // PH_INIT, PH_NEWTON, PH_FINAL evaluate at va
      }
      QR = rhs_lane(&sL, Md, Mi, scratch, src, ns, pj, pval, dst, P0, o.energy, a.rho ? a.rho[cell] : 0.);
      if (phase == PH_JAC) ++cnt[CNT_JAC_RHS];
      else ++cnt[CNT_RHS];
    }

    // =================== advance each solver to its next RHS request ===================
    enum : int { L_NONE, L_START_STEP, L_DRIVER_LOOP, L_JAC_COLUMN, L_AFTER_JAC, L_AFTER_FACT, L_NEWTON_TEST,
                 L_CORR_DONE, L_FINISH };
    int lab = L_NONE;
    if (!done) switch (phase) {
      case PH_INIT: {
        // MultiValueSolver::Solve, first call (:445-469)
        bool illegal = false;
        for (int k = 0; k < n; ++k) {
          const double yk = pva[k * ns];
          if (yk < lo_bound(k, NC, yminT) || yk > hi_bound(k, NC, ymaxT)) illegal = true;
        }
        if (illegal) { status = -9; lab = L_FINISH; break; }
        set_eps(pva, peps, n, ns, o.atol, o.rtol);
        double lo, hi;
        if (t0 != 0.) { lo = 100. * kMachEpsDouble * fabs(t0); hi = fabs(t0); }
        else { lo = kMachEpsDouble; hi = 1.e-4; }
        double h0 = 0.5 / (wrms(pf, peps, n, ns) + kMachEpsFloat);
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
          hf = 1.e+3 * kMachEpsDouble * fabs(h) * wrms(pf0, peps, n, ns) * double(n);
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
        for (int i = 0; i < n; ++i) pjac[(long)(i * n + jcol) * ns] = hInv * (pf[i * ns] - pf0[i * ns]);
        ++jcol;
        if (jcol < n) { lab = L_JAC_COLUMN; break; }
        ++cnt[CNT_JAC];
        factorized = 0;
        lab = L_AFTER_JAC;
        break;
      }
      case PH_NEWTON: {
        const double* v1 = Vp(1);
        for (int k = 0; k < n; ++k) DB(k) = pf[k * ns] * h - v1[k * ns] - pb[k * ns];
        lin_solve();
        for (int k = 0; k < n; ++k) pb[k * ns] += DB(k);
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
      default:
        status = -10;
        for (int k = 0; k < n; ++k) pva[k * ns] = pz[k * ns];
        lab = L_FINISH;
        break;
    }

    for (int pass = 0; pass < 2; ++pass) {
      if (pass == 1) {
        // warp-cooperative factorisations for the lanes that asked for one
        __syncwarp();
        unsigned fm = __ballot_sync(kFull, !done && phase == PH_FACT);
        while (fm) {
          const int ql = __ffs(fm) - 1;
          fm &= fm - 1;
          coop_factorize(ql, __shfl_sync(kFull, pendHr0, ql));
        }
        if (!done && phase == PH_FACT) {
          factorized = 1;
          ++cnt[CNT_FACT];
          lab = L_AFTER_FACT;
        } else {
          lab = L_NONE;
        }
      }
      // labels that need no RHS; a request or a finish is reached within a few hops
      for (int hop = 0; lab != L_NONE; ++hop) {
        if (hop >= 64) {
          status = -10;
          for (int k = 0; k < n; ++k) pva[k * ns] = pz[k * ns];
          lab = L_FINISH;
        }
        switch (lab) {
          case L_START_STEP: {
            // MultiValueSolver::Solve loop (:532-560) + DriverStep prologue (:753-776)
            if (numberOfSteps >= (unsigned)o.max_steps) {
              status = -1;
              for (int k = 0; k < n; ++k) pva[k * ns] = pz[k * ns];
              lab = L_FINISH;
              break;
            }
            set_eps(pz, peps, n, ns, o.atol, o.rtol);
            if (kMachEpsDouble * wrms(pz, peps, n, ns) > 1.) {
              status = -2;
              for (int k = 0; k < n; ++k) pva[k * ns] = pz[k * ns];
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
              rescale_z(pz, n, ns, p, hScale, NC, yminT, ymaxT);
              iterOrder = 0;
              odeHStatus = H_CONST;
            }
            h = hNextStep;
            hNordsieck = hNextStep;
            t = tInMeshPoint + h;
            if (t == tInMeshPoint) {
              status = -6;
              for (int k = 0; k < n; ++k) pva[k * ns] = pz[k * ns];
              t = tInMeshPoint;
              lab = L_FINISH;
              break;
            }
            predict(pz, pv, pvb, peps, n, ns, p, NC, yminT, ymaxT);
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
            if (yh + hJ > hi_bound(jcol, NC, ymaxT)) hJ = -hJ;
            phase = PH_JAC;
            lab = L_NONE;
            break;
          }
          case L_AFTER_JAC: {
            if (factorized && iterOrder == 0) factorized = 0;
            if (!factorized) {
              pendHr0 = h * c_gear_b.r[0][p - 1];
              phase = PH_FACT;
              lab = L_NONE;
              break;
            }
            lab = L_AFTER_FACT;
            break;
          }
          case L_AFTER_FACT: {
            const double* v1 = Vp(1);
            for (int k = 0; k < n; ++k) DB(k) = pf0[k * ns] * h - v1[k * ns];
            lin_solve();
            for (int k = 0; k < n; ++k) pb[k * ns] = DB(k);
            newtonK = 1;
            lab = L_NEWTON_TEST;
            break;
          }
          case L_NEWTON_TEST: {
            const double r0 = c_gear_b.r[0][p - 1];
            double s2 = 0.;
            for (int k = 0; k < n; ++k) {
              const double c = DB(k) * peps[k * ns];
              s2 += c * c;
            }
            const double cc = r0 * sqrt(s2 / double(n));
            if (cc < 1.) { convOK = 1; iterConvergence = newtonK; lab = L_CORR_DONE; break; }
            if (newtonK > 1 && cc > 2. * oldCC) { convOK = 0; iterConvergence = newtonK; lab = L_CORR_DONE; break; }
            oldCC = cc;
            const double* v0 = Vp(0);
            for (int k = 0; k < n; ++k) {
              double va = pb[k * ns] * r0 + v0[k * ns];
              const double lo = lo_bound(k, NC, yminT), hi = hi_bound(k, NC, ymaxT);
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
              ++cnt[CNT_CONVFAIL];
              if (iterConvergenceFailure >= 50u || fabs(h) <= 0.) {
                status = iterConvergenceFailure >= 50u ? -5 : -6;
                for (int k = 0; k < n; ++k) pva[k * ns] = pz[k * ns];
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
              const double r0 = c_gear_b.r[0][p - 1];
              double* v0 = Vp(0);
              double* v1 = Vp(1);
              for (int k = 0; k < n; ++k) {
                const double lo = lo_bound(k, NC, yminT), hi = hi_bound(k, NC, ymaxT);
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
                const double ri = c_gear_b.r[i][p - 1];
                double* vi = Vp(i);
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
            double hCur = c_gear_b.Ep[p] * wrms(Vp(p + 1), peps, n, ns);
            if (hCur > 1.) {
              iterErrorFailure++;
              ++cnt[CNT_ERRFAIL];
              if (iterErrorFailure >= 50u || fabs(h) <= 0.) {
                status = iterErrorFailure >= 50u ? -4 : -6;
                for (int k = 0; k < n; ++k) pva[k * ns] = pz[k * ns];
                t = tInMeshPoint;
                lab = L_FINISH;
                break;
              }
              hScaleMax = 1.;
              hCur = 0.8 * pow(1. / hCur, 1. / double(p + 1));
              hScale = hCur;
              if (p > 1u) {
                double hMinus = c_gear_b.Ep[p - 1] * wrms(Vp(p), peps, n, ns);
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
              // MethodGear::ConvergenceRate (:425-516) with the FP32 Jacobian
              if (iterErrorFailure > 0 || iterConvergenceFailure > 0) iterConvergenceRate = 0;
              if (iterConvergence > 1) {
                const double* v0 = Vp(0);
                const double* v1 = Vp(1);
                const double* z1 = Zp(1);
                double normd = 0., normf = 0.;
                for (int i = 0; i < n; ++i) {
                  double s = 0.;
                  for (int j = 0; j < n; ++j) s += (double)pjac[(long)(i * n + j) * ns] * (v0[j * ns] - pz[j * ns]);
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
                  hMinus = c_gear_b.Ep[p - 1] * wrms(Vp(p), peps, n, ns) + kMachEpsFloat;
                  hMinus = 1. / hMinus;
                  alfa1 = alfa2(p - 1) - .05;
                  hMinus = alfa1 * pow(hMinus, 1. / double(p));
                }
                hC = c_gear_b.Ep[p] * wrms(Vp(p + 1), peps, n, ns) + kMachEpsFloat;
                hC = 1. / hC;
                hC = alfa2(p) * pow(hC, 1. / double(p + 1));
                if (p < maximum_order && odeOrderStatus != O_DEC) {
                  hPlus = c_gear_b.Ep[p + 1] * wrms(Vp(p + 2), peps, n, ns) + kMachEpsFloat;
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
            for (unsigned i = 0; i <= p + 2; ++i) {
              const double* vi = Vp(i);
              double* zi = Zp(i);
              for (int k = 0; k < n; ++k) zi[k * ns] = vi[k * ns];
            }
            for (int k = 0; k < n; ++k) {
              double z0 = pz[k * ns];
              const double lo = lo_bound(k, NC, yminT), hi = hi_bound(k, NC, ymaxT);
              if (z0 < lo) z0 = lo;
              if (z0 > hi) z0 = hi;
              pz[k * ns] = z0;
            }
            numberOfSteps++;
            ++cnt[CNT_STEPS];
            if (tOut == t) {
              for (int k = 0; k < n; ++k) pva[k * ns] = pz[k * ns];
              lab = L_FINISH;
              break;
            }
            if (tOut < t) {
              // Interpolation (:687-706); the RHS at tOut then sets QR (:599-611)
              const double hp = (tOut - t) / hNordsieck;
              for (int k = 0; k < n; ++k) {
                double y = pz[k * ns];
                if (hp != 0.) {
                  double hr = 1.;
                  for (unsigned i = 1; i <= p; ++i) { hr *= hp; y += Zp(i)[k * ns] * hr; }
                  const double lo = lo_bound(k, NC, yminT), hi = hi_bound(k, NC, ymaxT);
                  if (y < lo) y = lo;
                  if (y > hi) y = hi;
                }
                pva[k * ns] = y;
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
            if (a.counters)
              for (int k = 0; k < NCNT; ++k) a.counters[(long)cell * NCNT + k] = cnt[k];
            phase = PH_FETCH;
            lab = L_NONE;
            break;
          }
          default:
            lab = L_NONE;
            break;
        }
      }
    }
  }
}

__host__ size_t batched_slot_doubles(const MechLayout& L, bool lu64) {
  (void)lu64;
  return (size_t)slot_layout(L).total;
}

size_t batched_smem_bytes(const MechLayout& L, bool lu64) {
  const size_t n = L.nc + 1;
  return ((L.bytes + 15u) & ~15u) + (size_t)4 * L.nc * kBT * sizeof(double) + n * kBT * sizeof(double) +
         ((n * n * kLS * (lu64 ? sizeof(double) : sizeof(float)) + 15) & ~(size_t)15) + n * kBT * sizeof(int) + 16;
}

int batched_threads_per_block() { return kBT; }

cudaError_t upload_gear_batched(const GearConsts& gc) {
  return cudaMemcpyToSymbol(c_gear_b, &gc, sizeof(GearConsts));
}

cudaError_t launch_batched(const MechLayout& L, const unsigned char* mech_gmem, const StepOptions& o,
                           const StepArgs& a, double* slots, long nslots, const int* order, int* queue, bool lu64,
                           int* err, cudaStream_t stream) {
  if (L.nc + 1 > 32) return cudaErrorInvalidValue;
  const size_t smem = batched_smem_bytes(L, lu64);
  const long blocks = nslots / kBT;
  if (blocks <= 0) return cudaErrorInvalidValue;
  const SlotLayout S = slot_layout(L);
  const long ns = nslots;
  double* gz = slots + (long)S.z * ns;
  double* gv = slots + (long)S.v * ns;
  double* gb = slots + (long)S.b * ns;
  double* gf = slots + (long)S.f * ns;
  double* gf0 = slots + (long)S.f0 * ns;
  double* gva = slots + (long)S.va * ns;
  double* gvb = slots + (long)S.vb * ns;
  double* geps = slots + (long)S.eps * ns;
  double* gr = slots + (long)S.r * ns;
  double* gjac = slots + (long)S.jac * ns;
  cudaError_t e;
  if (lu64) {
    e = cudaFuncSetAttribute(batched_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    batched_kernel<double><<<(unsigned)blocks, kBT, smem, stream>>>(L, mech_gmem, o, a, gz, gv, gb, gf, gf0, gva,
                                                                     gvb, geps, gr, gjac, ns, order, queue, err);
  } else {
    e = cudaFuncSetAttribute(batched_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    batched_kernel<float><<<(unsigned)blocks, kBT, smem, stream>>>(L, mech_gmem, o, a, gz, gv, gb, gf, gf0, gva,
                                                                    gvb, geps, gr, gjac, ns, order, queue, err);
  }
  return cudaGetLastError();
}

cudaError_t batched_occupancy(const MechLayout& L, bool lu64, int* blocks_per_sm) {
  const size_t smem = batched_smem_bytes(L, lu64);
  cudaError_t e;
  if (lu64) {
    e = cudaFuncSetAttribute(batched_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, batched_kernel<double>, kBT, smem);
  }
  e = cudaFuncSetAttribute(batched_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, batched_kernel<float>, kBT, smem);
}

// ---------------------------------------------------------------------------
// No-allocation variant.  Some callers cannot allocate device memory when they
// advance the chemistry: a solver that hands all free device memory to its own
// pool allocator at start-up, or one that must not let cudaMalloc/cudaFree
// (which synchronise the device) into its time-step loop.  For them the lane
// kernel above runs with its slot scratch in this fixed array instead of a
// context buffer; the number of slots is whatever fits, so any cell count is
// served (cells are taken from the queue), just with fewer cells in flight.
//
// Layout: bytes [0, 256) hold the control words (int queue counter, int error
// flags), zeroed by every call; the slots start at byte 256.  Every call on a
// device shares the array and the array keeps the last call's contents, so
// calls that overlap on the GPU (two streams, two host threads) race: callers
// serialise them.  Every GPU that loads this part of the library holds the
// array until the process exits.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[64] = {};
}  // namespace

// Device address of the scratch array on the current device (set up once per
// device; host code cannot use the array's name as a device address).
static cudaError_t noalloc_scratch(int device, unsigned char** out) {
  if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_noalloc_mutex);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[device] = p;
  }
  *out = (unsigned char*)g_noalloc_ptr[device];
  return cudaSuccess;
}

// Loads this file's kernels and the scratch array on `device` (the current
// device) and looks up the array's address.  CUDA loads modules and kernels
// lazily, and loading commits device memory (kernel code, and the 16 MiB
// array itself); doing it when a mechanism is loaded keeps every such
// commitment ahead of a caller that then hands the free memory to its pool.
cudaError_t batched_noalloc_prepare(int device) {
  cudaFuncAttributes fa{};
  cudaError_t e = cudaFuncGetAttributes(&fa, batched_kernel<double>);
  if (e != cudaSuccess) return e;
  e = cudaFuncGetAttributes(&fa, batched_kernel<float>);
  if (e != cudaSuccess) return e;
  unsigned char* base = nullptr;
  return noalloc_scratch(device, &base);
}

long batched_noalloc_slots(const MechLayout& L, bool lu64, int sm_count) {
  int bps = 0;
  if (batched_occupancy(L, lu64, &bps) != cudaSuccess || bps <= 0) return -1;
  const size_t per_block = batched_slot_doubles(L, lu64) * sizeof(double) * kBT;
  const long fit = (long)((kNoAllocScratchBytes - 256) / per_block);
  const long full = (long)sm_count * bps;
  const long blocks = fit < full ? fit : full;
  return blocks * kBT;   // 0 when not even one block of slots fits
}

cudaError_t launch_batched_noalloc(const MechLayout& L, const unsigned char* mech_gmem, const StepOptions& o,
                                   const StepArgs& a, bool lu64, int device, long nslots, int* host_flags,
                                   cudaStream_t stream) {
  if (nslots < kBT) return cudaErrorInvalidValue;
  unsigned char* base = nullptr;
  cudaError_t e = noalloc_scratch(device, &base);
  if (e != cudaSuccess) return e;
  int* queue = (int*)base;
  int* err = queue + 1;
  double* slots = (double*)(base + 256);
  e = cudaMemsetAsync(base, 0, 256, stream);   // the queue counter and the error flags start at zero
  if (e != cudaSuccess) return e;
  e = launch_batched(L, mech_gmem, o, a, slots, nslots, nullptr, queue, lu64, err, stream);
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(host_flags, err, sizeof(int), cudaMemcpyDeviceToHost, stream);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(stream);
}

}  // namespace lsg
