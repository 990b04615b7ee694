// Common device helpers: constants, warp reductions in a fixed order, the
// bulk (TMA engine) staging of the mechanism table into shared memory.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "lsg_mech.h"

namespace lsg {

// math/OpenSMOKEFunctions.hpp:60-87 and math/OpenSMOKEStdInclude.h:53-55
constexpr double kMachEpsDouble = 2.220446049250313e-16;
constexpr double kMachEpsFloat = 1.1920928955078125e-07;   // (double)1.192092896e-07F
constexpr double kTinyFloat = 1.1754943508222875e-38;      // (double)1.175494351e-38F
constexpr double kRgas = 8314.4621;                        // J/kmol/K, math/PhysicalConstants.h:24
constexpr unsigned kFull = 0xffffffffu;

// Error flags written to the per-call device error word.
enum : int {
  kErrNone = 0,
  kErrStageTimeout = 1,     // bulk copy of the mechanism did not complete in time
  kErrBadSize = 2,
  kErrQueueTimeout = 4,
  kErrTensorCoreWait = 8,   // a tensor-core MMA did not report completion within the wait limit
};

// Sum of v over lanes 0..n-1, added strictly in lane order (the reference's
// sequential loops).  Every lane receives the result.
__device__ __forceinline__ double seq_sum(double v, int n) {
  double s = 0.;
  for (int i = 0; i < n; ++i) s += __shfl_sync(kFull, v, i);
  return s;
}

// Rate constant of a pressure-logarithmic (PLOG) reaction at T and P
// (PressureLogarithmicRateExpression::KineticConstant,
// PressureLogarithmicRateExpression.hpp:104-119): the first or last point
// outside the tabulated pressures, else ln k interpolated linearly in ln P
// between the two points that bracket P.
static __device__ __noinline__ double plog_k(const MechView& M, const MechLayout& L, int slot, double T, double logT,
                                         double P) {
  const int a = M.I(L.plog_ptr)[slot], b = M.I(L.plog_ptr)[slot + 1];
  const double* p = M.D(L.plog_p);
  const double* lnA = M.D(L.plog_lnA);
  const double* be = M.D(L.plog_beta);
  const double* er = M.D(L.plog_eor);
  if (P <= p[a]) return exp(lnA[a] + be[a] * logT - er[a] / T);
  if (P >= p[b - 1]) return exp(lnA[b - 1] + be[b - 1] * logT - er[b - 1] / T);
  int i = a;
  for (; i < b - 1; ++i)
    if (P < p[i + 1]) break;
  const double* lnp = M.D(L.plog_lnp);
  const double kA = lnA[i] + be[i] * logT - er[i] / T;
  const double kB = lnA[i + 1] + be[i + 1] * logT - er[i + 1] / T;
  return exp(kA + (kB - kA) * (log(P) - lnp[i]) / (lnp[i + 1] - lnp[i]));
}

// PLOG interpolation of points q0 .. q1 - 1 of a table (PressureLogarithmicRateExpression.hpp:104-119 and
// ExtendedPressureLogarithmicRateExpression.hpp:181-202): the first or last point outside the table, else
// ln k linear in ln P between the bracketing points.
static __device__ __forceinline__ double plog_points(const double* p, const double* lnp, const double* lnA,
                                                     const double* be, const double* er, int q0, int q1, double T,
                                                     double logT, double P) {
  if (P <= p[q0]) return exp(lnA[q0] + be[q0] * logT - er[q0] / T);
  if (P >= p[q1 - 1]) return exp(lnA[q1 - 1] + be[q1 - 1] * logT - er[q1 - 1] / T);
  int i = q0;
  for (; i < q1 - 1; ++i)
    if (P < p[i + 1]) break;
  const double kA = lnA[i] + be[i] * logT - er[i] / T;
  const double kB = lnA[i + 1] + be[i + 1] * logT - er[i + 1] / T;
  return exp(kA + (kB - kA) * (log(P) - lnp[i]) / (lnp[i + 1] - lnp[i]));
}

// Extended PLOG (PLOGMX / PLOGSP; KineticsMap_CHEMKIN.hpp:1662-1670 with
// ExtendedPressureLogarithmicRateExpression::KineticConstant, :162-179): the
// rate constant of slot `slot` at T, P and the concentrations conc(k):
//   k = (sum over bath species c_s k_s + (cTot - sum c_s) k_mixture) / cTot,
// each k a PLOG interpolation of that bath's table; cTot the kinetics map's
// sum of the concentrations.  Replaces the reaction's Arrhenius constant.
template <class Conc>
__device__ double xplog_k(const MechView& M, const MechLayout& L, int slot, double T, double logT, double P,
                          double cTot, Conc conc) {
  const int* bp = M.I(L.xplog_bath_ptr);
  const int* bs = M.I(L.xplog_bath_sp);
  const int* qp = M.I(L.xplog_ptr);
  double rest = cTot;
  for (int b = bp[slot]; b < bp[slot + 1]; ++b)
    if (bs[b] != -1) rest -= conc(bs[b]);
  double kc = 0.;
  for (int b = bp[slot]; b < bp[slot + 1]; ++b) {
    const double kb = plog_points(M.D(L.xplog_p), M.D(L.xplog_lnp), M.D(L.xplog_lnA), M.D(L.xplog_beta),
                                  M.D(L.xplog_eor), qp[b], qp[b + 1], T, logT, P);
    kc += (bs[b] != -1 ? conc(bs[b]) : rest) * kb;
  }
  return kc / cTot;
}

// Extended fall-off (LOWMX / LOWSP; KineticsMap_CHEMKIN.hpp:1672-1681 with
// ExtendedFallOff::KineticConstant, ExtendedFallOff.hpp:170-240): per bath
// k_inf (Pr / (1 + Pr)) F with the bath's own low-pressure limit k0 and its
// Lindemann, Troe or SRI form, M from the reaction's efficiencies, the baths
// weighted by concentration as in the extended PLOG.  Replaces the reaction's
// modified rate constant.
template <class Conc>
__device__ double xfo_k(const MechView& M, const MechLayout& L, int slot, double T, double cTot, Conc conc) {
  const double* ki = M.D(L.xfo_kinf) + 3 * slot;
  const double kInf = ki[0] * pow(T, ki[1]) * exp(-ki[2] / T);
  const int* tp = M.I(L.xfo_tb_ptr);
  const int* ts = M.I(L.xfo_tb_sp);
  const double* te = M.D(L.xfo_tb_eff);
  double Mc = cTot;
  for (int q = tp[slot]; q < tp[slot + 1]; ++q) Mc += te[q] * conc(ts[q]);
  const int* bp = M.I(L.xfo_bath_ptr);
  const int* bs = M.I(L.xfo_bath_sp);
  const int* ty = M.I(L.xfo_type);
  const int* pp = M.I(L.xfo_par_ptr);
  double rest = cTot;
  for (int b = bp[slot]; b < bp[slot + 1]; ++b)
    if (bs[b] != -1) rest -= conc(bs[b]);
  double kc = 0.;
  for (int b = bp[slot]; b < bp[slot + 1]; ++b) {
    const double* lo = M.D(L.xfo_low) + 3 * b;
    const double k0 = lo[0] * pow(T, lo[1]) * exp(-lo[2] / T);
    const double Pr = k0 / kInf * Mc;
    const double* t = M.D(L.xfo_par) + pp[b];
    const int nt = pp[b + 1] - pp[b];
    double F = 1.;
    if (ty[b] == 1) {
      double Fcent = (1. - t[0]) * exp(-T / t[1]) + t[0] * exp(-T / t[2]);
      if (nt == 4) Fcent += exp(-t[3] / T);
      double logFcent = -300.;
      if (Fcent > 1e-300) logFcent = log10(Fcent);
      double q;
      if (Pr > 1.e-32) {
        const double cc = -0.4 - 0.67 * logFcent;
        const double nn = 0.75 - 1.27 * logFcent;
        const double e = log10(Pr) + cc;
        q = e / (nn - 0.14 * e);
      } else {
        q = 1. / 0.14;
      }
      F = pow(10., logFcent / (1. + q * q));
    } else if (ty[b] == 2) {
      const double l = log10(Pr);
      const double X = 1. / (1. + l * l);
      F = pow(t[0] * exp(-t[1] / T) + exp(-T / t[2]), X);
      if (nt == 5) F *= t[3] * pow(T, t[4]);
    }
    kc += (bs[b] != -1 ? conc(bs[b]) : rest) * (kInf * (Pr / (1. + Pr)) * F);
  }
  return kc / cTot;
}

// Rate constant of a Chebyshev reaction at T and P
// (ChebyshevPolynomialRateExpression::KineticConstant, :93-114, with
// Phi(n, x) = cos((n - 1) acos(x)), :187-190): 10^(sum_nm a_nm phi_n(T~) phi_m(P~))
// times the unit conversion, T~ and P~ the reduced inverse temperature and
// log10 pressure.  Outside the limits acos is undefined, as in the reference.
static __device__ __noinline__ double cheb_k(const MechView& M, const MechLayout& L, int slot, double T, double P) {
  const int N = M.I(L.cheb_nm)[2 * slot], Mm = M.I(L.cheb_nm)[2 * slot + 1];
  const double* a = M.D(L.cheb_coef) + M.I(L.cheb_ptr)[slot];
  const double* lim = M.D(L.cheb_lim) + 5 * slot;
  const double Tmin = lim[0], Tmax = lim[1], lPmin = lim[2], lPmax = lim[3];
  const double Tt = (2. / T - 1. / Tmin - 1. / Tmax) / (1. / Tmax - 1. / Tmin);
  const double Pt = (2. * log10(P) - lPmin - lPmax) / (lPmax - lPmin);
  const double aT = acos(Tt), aP = acos(Pt);
  double sum = 0.;
  for (int n = 0; n < N; ++n) {
    const double phn = cos(double(n) * aT);
    for (int m = 0; m < Mm; ++m) sum += a[n * Mm + m] * phn * cos(double(m) * aP);
  }
  return pow(10., sum) * lim[4];
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Stage `bytes` (multiple of 16, both addresses 16-byte aligned) from global
// to shared memory with one-dimensional bulk copies issued by thread 0 and
// completed on an mbarrier.  Waits are bounded; on timeout the block's
// error flag is raised and false is returned (the caller must then not use
// the shared copy).  Must be called by all threads of the block.
__device__ inline bool stage_bulk(void* smem_dst, const void* gsrc, uint32_t bytes, uint64_t* mbar, int* err) {
  const uint32_t bar = smem_u32(mbar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
    const uint32_t dst = smem_u32(smem_dst);
    const uint32_t chunk = 32768;   // several copies, each a multiple of 16 bytes
    for (uint32_t off = 0; off < bytes; off += chunk) {
      const uint32_t n = (bytes - off) < chunk ? (bytes - off) : chunk;
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst + off),
          "l"((const char*)gsrc + off), "r"(n), "r"(bar)
          : "memory");
    }
  }
  uint32_t done = 0;
  for (long it = 0; it < (1L << 22); ++it) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar)
        : "memory");
    if (done) break;
  }
  const int ok = __syncthreads_and(done ? 1 : 0);
  if (!ok && threadIdx.x == 0) atomicOr(err, kErrStageTimeout);
  return ok != 0;
}

// Net stoichiometric coefficient of species s in reaction k, formed as the
// reference's DRG constructor forms it: products added first, then reactants
// subtracted (DRG.hpp:45-110).  Zero when s does not take part.
__device__ __forceinline__ double drg_net_nu(const MechView& M, const MechLayout& L, int k, int s) {
  const int* rp = M.I(L.reac_ptr);
  const int* rsp = M.I(L.reac_sp);
  const double* rnu = M.D(L.reac_nu);
  const int* pp = M.I(L.prod_ptr);
  const int* psp = M.I(L.prod_sp);
  const double* pnu = M.D(L.prod_nu);
  double v = 0.;
  for (int q = pp[k]; q < pp[k + 1]; ++q)
    if (psp[q] == s) v += pnu[q];
  for (int q = rp[k]; q < rp[k + 1]; ++q)
    if (rsp[q] == s) v -= rnu[q];
  return v;
}

}  // namespace lsg
