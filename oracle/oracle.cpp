// CPU oracle for the laminarSMOKE reaction step -- TEST INFRASTRUCTURE ONLY.
//
// This file restates, in plain FP64 C++, the reference's constant-pressure
// batch-reactor chemistry step.  It is used by the tests (as the parity
// checker), by __graft_entry__.smoke() and by bench.py's CPU baseline leg,
// and by nothing else: the product path (the CUDA library) never calls it.
//
// Parity status: UNPINNED.  The reference ships no tests, fixtures or golden
// vectors for this path, and its code cannot be compiled here (it needs
// Eigen 3.3.7, Boost 1.69, RapidXML and OpenFOAM, none of which is present).
// The restatement follows the reference line by line instead; each function
// below names the file:line it follows (paths relative to
// solvers/openSMOKEpp4laminarSMOKE unless they start with solvers/).
//
// Build: oracle/Makefile (g++ -O2 -ffp-contract=off -fopenmp).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cfloat>
#include <string>
#include <vector>
#include <algorithm>
#include <map>
#include <stdexcept>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// math/OpenSMOKEFunctions.hpp:60-87, math/OpenSMOKEStdInclude.h:53-55
static const double MACH_EPS_DOUBLE = 2.220446049250313e-16;      // MachEps()
static const double MACH_EPS_FLOAT = (double)1.192092896e-07F;      // MachEpsFloat()
static const double TINY_FLOAT = (double)1.175494351e-38F;         // OPENSMOKE_TINY_FLOAT
static const double R_J_KMOL = 8314.4621;                            // math/PhysicalConstants.h:24

// ---------------------------------------------------------------------------
// Packed mechanism (the blob written by laminarsmoke_b200/mech/blob.py)
// ---------------------------------------------------------------------------
struct Mech {
  int nc = 0, nr = 0;
  std::map<std::string, std::vector<double>> f;
  std::map<std::string, std::vector<int>> i;
  const std::vector<double>& F(const char* k) const {
    auto it = f.find(k);
    if (it == f.end()) throw std::runtime_error(std::string("missing array ") + k);
    return it->second;
  }
  const std::vector<int>& I(const char* k) const {
    auto it = i.find(k);
    if (it == i.end()) throw std::runtime_error(std::string("missing array ") + k);
    return it->second;
  }
};

static Mech* load_blob(const unsigned char* p, size_t n) {
  if (n < 16 || std::memcmp(p, "LSMECH01", 8) != 0) return nullptr;
  uint32_t na; std::memcpy(&na, p + 8, 4);
  size_t pos = 16;
  Mech* m = new Mech();
  for (uint32_t a = 0; a < na; ++a) {
    if (pos + 48 > n) { delete m; return nullptr; }
    char name[33]; std::memcpy(name, p + pos, 32); name[32] = 0;
    uint32_t code; uint64_t count;
    std::memcpy(&code, p + pos + 32, 4); std::memcpy(&count, p + pos + 40, 8);
    pos += 48;
    if (code > 1) { delete m; return nullptr; }
    const size_t item = code == 0 ? 8 : 4;
    if (count > (n - pos) / item) { delete m; return nullptr; }   // no overflow of item * count
    const size_t nb = item * count;
    if (code == 0) { std::vector<double> v(count); std::memcpy(v.data(), p + pos, nb); m->f[name] = v; }
    else { std::vector<int> v(count); std::memcpy(v.data(), p + pos, nb); m->i[name] = v; }
    pos += nb + ((8 - nb % 8) % 8);
  }
  m->nc = m->I("dims")[0];
  m->nr = m->I("dims")[1];
  // Forward rate-law orders (ReactionPolicy_CHEMKIN reactant_lambda_): the FORD lists when the mechanism
  // has them, else the reactant coefficients (ReactionPolicy_CHEMKIN.hpp:380-381).
  if (!m->f.count("ford_val")) {
    m->i["ford_ptr"] = m->I("reac_ptr");
    m->i["ford_species"] = m->I("reac_species");
    m->f["ford_val"] = m->F("reac_nu");
  }
  return m;
}

// ---------------------------------------------------------------------------
// Reactor right-hand side with the reference's per-temperature caching.
//   solvers/laminarSMOKE/unsteady/BatchReactorHomogeneousConstantPressure.H:175-223
//   maps/ThermodynamicsMap_CHEMKIN.hpp:158-164, 429-520
//   maps/KineticsMap_CHEMKIN.hpp:271-297, 1181-1398, 1496-1550, 1683-1768, 1956-1964
//   maps/StoichiometricMap.hpp:512-598, 656-729, 916-1001
// ---------------------------------------------------------------------------
struct Reactor {
  const Mech& m;
  int NC, NR;
  double P0 = 101325.;
  double rho0 = 0.;   // > 0: constant-volume reactor of this density (BatchReactorHomogeneousConstantVolume.H)
  double P_ = 101325.;   // the kinetics map's pressure: P0, or cTot R T at constant volume
  bool energy = true;
  double QR = 0.;
  // thermo map
  std::vector<double> cp, h, s;
  // kinetics map caches
  double T_ = 0., T_old_ = 0.;
  bool arr_recalc = true, hs_recalc = true;
  std::vector<double> kArr, uKeq, kRev, kInf, logFcent, rdh, rds, kMod, fwd, rev, net, corr;
  std::vector<double> x, c, R;
  std::vector<double> Mtb;   // M of each third-body reaction at the last reaction_rates()
  long long n_calls = 0;

  explicit Reactor(const Mech& mech) : m(mech), NC(mech.nc), NR(mech.nr) {
    cp.resize(NC); h.resize(NC); s.resize(NC);
    kArr.resize(NR); kMod.resize(NR); fwd.resize(NR); rev.resize(NR); net.resize(NR);
    rdh.resize(NR); rds.resize(NR);
    uKeq.resize(m.I("rev_thermo").size());
    kRev.resize(m.I("rev_explicit").size());
    kInf.resize(m.I("fo_rxn").size()); logFcent.resize(kInf.size()); corr.resize(kInf.size());
    x.resize(NC); c.resize(NC); R.resize(NC);
    Mtb.resize(m.I("tb_rxn").size());
  }

  // KineticsMap_CHEMKIN::FallOffReactionsCorrection (:1552-1610): the fall-off factor of slot k at the
  // concentrations cc, with the constants of the last reaction_rates()
  double falloff_correction(int k, double cTot, const double* cc) const {
    const auto& fr = m.I("fo_rxn"); const auto& fty = m.I("fo_type"); const auto& fsg = m.I("fo_single");
    const auto& fp = m.I("fo_ptr"); const auto& fs = m.I("fo_species"); const auto& fe = m.F("fo_eff_m1");
    const auto& fd = m.F("fo_d"); const auto& fee = m.F("fo_e");
    double M;
    if (fsg[k] < 0) {
      M = cTot;
      for (int q = fp[k]; q < fp[k + 1]; ++q) M += cc[fs[q]] * fe[q];
    } else {
      M = cc[fsg[k]] + 1.e-16;
    }
    const int j = fr[k];
    const double Pr = kArr[j] * M / kInf[k];
    double wF = 1.;
    if (fty[k] == 1) {
      if (Pr > 1.e-32) {
        const double nTroe = 0.75 - 1.27 * logFcent[k];
        const double cTroe = -0.4 - 0.67 * logFcent[k];
        const double sTroe = std::log10(Pr) + cTroe;
        const double q = sTroe / (nTroe - 0.14 * sTroe);
        wF = std::pow(10., logFcent[k] / (1. + q * q));
      } else {
        const double q = 1. / 0.14;
        wF = std::pow(10., logFcent[k] / (1. + q * q));
      }
    } else if (fty[k] == 2) {
      double xSRI = 0.;
      if (Pr > 1.e-32) {
        const double l = std::log10(Pr);
        xSRI = 1. / (1. + l * l);
      }
      wF = std::pow(logFcent[k], xSRI) * fd[k];
      if (fee[k] != 0.) wF *= std::pow(T_, fee[k]);
    }
    return kInf[k] * (Pr / (1. + Pr)) * wF / kArr[j];
  }

  // ThermodynamicsMap_CHEMKIN::cp_over_R (:436-454)
  void cp_over_R(double T) {
    const auto& HT = m.F("cp_ht"); const auto& LT = m.F("cp_lt"); const auto& TM = m.F("t_mid");
    const double T2 = T * T, T3 = T2 * T, T4 = T3 * T;
    int j = 0;
    for (int k = 0; k < NC; ++k) {
      cp[k] = (T > TM[k]) ? HT[j] + T * HT[j + 1] + T2 * HT[j + 2] + T3 * HT[j + 3] + T4 * HT[j + 4]
                          : LT[j] + T * LT[j + 1] + T2 * LT[j + 2] + T3 * LT[j + 3] + T4 * LT[j + 4];
      j += 5;
    }
  }
  // ThermodynamicsMap_CHEMKIN::h_over_RT (:456-475)
  void h_over_RT(double T) {
    const auto& HT = m.F("dh_ht"); const auto& LT = m.F("dh_lt"); const auto& TM = m.F("t_mid");
    const double T2 = T * T, T3 = T2 * T, T4 = T3 * T, uT = 1. / T;
    int j = 0;
    for (int k = 0; k < NC; ++k) {
      h[k] = (T > TM[k]) ? HT[j] + T * HT[j + 1] + T2 * HT[j + 2] + T3 * HT[j + 3] + T4 * HT[j + 4] + uT * HT[j + 5]
                         : LT[j] + T * LT[j + 1] + T2 * LT[j + 2] + T3 * LT[j + 3] + T4 * LT[j + 4] + uT * LT[j + 5];
      j += 6;
    }
  }
  // ThermodynamicsMap_CHEMKIN::s_over_R (:477-496)
  void s_over_R(double T) {
    const auto& HT = m.F("ds_ht"); const auto& LT = m.F("ds_lt"); const auto& TM = m.F("t_mid");
    const double logT = std::log(T), T2 = T * T, T3 = T2 * T, T4 = T3 * T;
    int j = 0;
    for (int k = 0; k < NC; ++k) {
      s[k] = (T > TM[k]) ? HT[j] * logT + T * HT[j + 1] + T2 * HT[j + 2] + T3 * HT[j + 3] + T4 * HT[j + 4] + HT[j + 5]
                         : LT[j] * logT + T * LT[j + 1] + T2 * LT[j + 2] + T3 * LT[j + 3] + T4 * LT[j + 4] + LT[j + 5];
      j += 6;
    }
  }

  // StoichiometricMap::ReactionEnthalpyAndEntropy (:916-1001): per reaction the
  // species contributions are added in species order, reactant side first.
  void reaction_h_s() {
    const auto& rp = m.I("reac_ptr"); const auto& rs = m.I("reac_species"); const auto& rn = m.F("reac_nu");
    const auto& pp = m.I("prod_ptr"); const auto& ps = m.I("prod_species"); const auto& pn = m.F("prod_nu");
    for (int j = 0; j < NR; ++j) {
      double dh = 0., ds = 0.;
      int a = rp[j], b = pp[j];
      while (a < rp[j + 1] || b < pp[j + 1]) {
        int sa = a < rp[j + 1] ? rs[a] : 1 << 30;
        int sb = b < pp[j + 1] ? ps[b] : 1 << 30;
        if (sa <= sb) {  // reactant contribution of species sa
          const double nu = rn[a];
          dh -= contrib(nu, h[sa]); ds -= contrib(nu, s[sa]); ++a;
        } else {
          const double nu = pn[b];
          dh += contrib(nu, h[sb]); ds += contrib(nu, s[sb]); ++b;
        }
      }
      rdh[j] = dh; rds[j] = ds;
    }
  }
  static double contrib(double nu, double v) {
    if (nu == 1.) return v;
    if (nu == 2.) return v + v;
    if (nu == 3.) return v + v + v;
    if (nu == 0.5) return 0.5 * v;
    return nu * v;
  }

  // KineticsMap_CHEMKIN::SetTemperature (:271-287)
  void kin_set_T(double T) {
    T_old_ = T_; T_ = T;
    if (std::fabs(T_ - T_old_) / T_ > 0.) { arr_recalc = true; hs_recalc = true; }
  }

  // KineticsMap_CHEMKIN::KineticConstants (:1181-1386)
  void kinetic_constants() {
    const double T = T_, uT = 1. / T, logT = std::log(T);
    const double Patm_over_RT = 101325. / R_J_KMOL / T;
    const double log_Patm_over_RT = std::log(Patm_over_RT);
    if (hs_recalc) { s_over_R(T); reaction_h_s(); hs_recalc = false; }
    if (arr_recalc) {
      const auto& lnA = m.F("lnA"); const auto& beta = m.F("beta"); const auto& eor = m.F("e_over_r");
      const auto& sgn = m.I("a_sign");
      for (int j = 0; j < NR; ++j) kArr[j] = std::exp(lnA[j] + beta[j] * logT - eor[j] * uT);
      for (int j = 0; j < NR; ++j) if (sgn[j] < 0) kArr[j] *= -1.;
      const auto& rth = m.I("rev_thermo"); const auto& dnu = m.F("delta_nu");
      for (size_t k = 0; k < rth.size(); ++k) {
        const int j = rth[k];
        uKeq[k] = std::exp(-rds[j] + rdh[j] - log_Patm_over_RT * dnu[j]);
      }
      const auto& lr = m.F("lnA_rev"); const auto& br = m.F("beta_rev"); const auto& er = m.F("e_over_r_rev");
      for (size_t k = 0; k < kRev.size(); ++k) kRev[k] = std::exp(lr[k] + br[k] * logT - er[k] * uT);
      const auto& fl = m.F("fo_lnA"); const auto& fb = m.F("fo_beta"); const auto& fe = m.F("fo_e_over_r");
      const auto& ft = m.I("fo_type");
      const auto& a = m.F("fo_a"); const auto& b = m.F("fo_b"); const auto& cc = m.F("fo_c"); const auto& d = m.F("fo_d");
      for (size_t k = 0; k < kInf.size(); ++k) kInf[k] = std::exp(fl[k] + fb[k] * logT - fe[k] * uT);
      for (size_t k = 0; k < kInf.size(); ++k) {
        if (ft[k] == 1) {
          double v = (d[k] != 0.) ? (1. - a[k]) * std::exp(-T / b[k]) + a[k] * std::exp(-T / cc[k]) + std::exp(-d[k] / T)
                                  : (1. - a[k]) * std::exp(-T / b[k]) + a[k] * std::exp(-T / cc[k]);
          logFcent[k] = (v < 1.e-300) ? -300. : std::log10(v);
        } else if (ft[k] == 2) {
          logFcent[k] = a[k] * std::exp(-b[k] / T) + std::exp(-T / cc[k]);
        }
      }
      arr_recalc = false;
    }
    // pressure-logarithmic reactions, every call: their k depends on P as well
    // (KineticsMap_CHEMKIN.hpp:1341-1348, PressureLogarithmicRateExpression.hpp:104-119)
    if (m.f.count("plog_p")) {
      const auto& prx = m.I("plog_rxn"); const auto& pptr = m.I("plog_ptr");
      const auto& pp = m.F("plog_p"); const auto& lnp = m.F("plog_lnp"); const auto& lA = m.F("plog_lnA");
      const auto& pb = m.F("plog_beta"); const auto& pe = m.F("plog_eor");
      for (size_t k = 0; k < prx.size(); ++k) {
        const int a = pptr[k], b = pptr[k + 1];
        double kk;
        if (P_ <= pp[a]) kk = std::exp(lA[a] + pb[a] * std::log(T) - pe[a] / T);
        else if (P_ >= pp[b - 1]) kk = std::exp(lA[b - 1] + pb[b - 1] * std::log(T) - pe[b - 1] / T);
        else {
          int i = a;
          for (; i < b - 1; ++i) if (P_ < pp[i + 1]) break;
          const double kA = lA[i] + pb[i] * std::log(T) - pe[i] / T;
          const double kB = lA[i + 1] + pb[i + 1] * std::log(T) - pe[i + 1] / T;
          kk = std::exp(kA + (kB - kA) * (std::log(P_) - lnp[i]) / (lnp[i + 1] - lnp[i]));
        }
        kArr[prx[k]] = kk;
      }
    }
    // Chebyshev reactions, every call (KineticsMap_CHEMKIN.hpp:1332-1339,
    // ChebyshevPolynomialRateExpression.hpp:93-114 and :187-190)
    if (m.f.count("cheb_coef")) {
      const auto& crx = m.I("cheb_rxn"); const auto& cnm = m.I("cheb_nm"); const auto& cptr = m.I("cheb_ptr");
      const auto& cco = m.F("cheb_coef"); const auto& clim = m.F("cheb_lim");
      for (size_t k = 0; k < crx.size(); ++k) {
        const int N = cnm[2 * k], Mm = cnm[2 * k + 1];
        const double* lim = &clim[5 * k];
        const double Ttilde = (2. / T - 1. / lim[0] - 1. / lim[1]) / (1. / lim[1] - 1. / lim[0]);
        const double Ptilde = (2. * std::log10(P_) - lim[2] - lim[3]) / (lim[3] - lim[2]);
        std::vector<double> phn(N), phm(Mm);
        for (int n = 1; n <= N; ++n) phn[n - 1] = std::cos(double(n - 1) * std::acos(Ttilde));
        for (int mm = 1; mm <= Mm; ++mm) phm[mm - 1] = std::cos(double(mm - 1) * std::acos(Ptilde));
        double sum = 0.;
        for (int n = 0; n < N; ++n)
          for (int mm = 0; mm < Mm; ++mm) sum += cco[cptr[k] + n * Mm + mm] * phn[n] * phm[mm];
        kArr[crx[k]] = std::pow(10., sum) * lim[4];
      }
    }
    kMod = kArr;
  }

  // KineticsMap_CHEMKIN::ReactionRates (:1683-1768) and FallOffReactions (:1496-1550)
  // ExtendedPressureLogarithmicRateExpression::KineticConstant(index, T, P) (:181-202): the PLOG
  // interpolation of one bath's table q0 .. q1 - 1
  double xplog_k(int q0, int q1, double T, double P) const {
    const auto& pp = m.F("xplog_p"); const auto& lnp = m.F("xplog_lnp"); const auto& lA = m.F("xplog_lnA");
    const auto& pb = m.F("xplog_beta"); const auto& pe = m.F("xplog_eor");
    const int n = q1 - q0;
    if (P <= pp[q0]) return std::exp(lA[q0] + pb[q0] * std::log(T) - pe[q0] / T);
    if (P >= pp[q1 - 1]) return std::exp(lA[q1 - 1] + pb[q1 - 1] * std::log(T) - pe[q1 - 1] / T);
    int i = 0;
    for (i = 0; i < n - 1; ++i)
      if (P < pp[q0 + i + 1]) break;
    const int a = q0 + i, b = a + 1;
    const double ln_kA = lA[a] + pb[a] * std::log(T) - pe[a] / T;
    const double ln_kB = lA[b] + pb[b] * std::log(T) - pe[b] / T;
    return std::exp(ln_kA + (ln_kB - ln_kA) * (std::log(P) - lnp[a]) / (lnp[b] - lnp[a]));
  }

  // KineticsMap_CHEMKIN::ExtendedPressureLogReactions (:1662-1670) with
  // ExtendedPressureLogarithmicRateExpression::KineticConstant(T, P, cTot, c) (:162-179):
  // k = (sum over bath species c_s k_s + (cTot - sum c_s) k_mixture) / cTot replaces the Arrhenius k
  void extended_plog(double cTot) {
    if (!m.i.count("xplog_rxn")) return;
    const auto& xr = m.I("xplog_rxn"); const auto& bp = m.I("xplog_bath_ptr");
    const auto& bs = m.I("xplog_bath_sp"); const auto& qp = m.I("xplog_ptr");
    for (size_t k = 0; k < xr.size(); ++k) {
      double rest = cTot;
      for (int b = bp[k]; b < bp[k + 1]; ++b) if (bs[b] != -1) rest -= c[bs[b]];
      double kc = 0.;
      for (int b = bp[k]; b < bp[k + 1]; ++b) {
        const double kb = xplog_k(qp[b], qp[b + 1], T_, P_);
        kc += (bs[b] != -1 ? c[bs[b]] : rest) * kb;
      }
      kc /= cTot;
      kArr[xr[k]] = kc;
      kMod[xr[k]] = kc;
    }
  }

  // KineticsMap_CHEMKIN::ExtendedFallOffReactions (:1672-1681) with ExtendedFallOff::KineticConstant
  // (ExtendedFallOff.hpp:170-240): per bath k = k_inf Pr / (1 + Pr) F with its own low-pressure limit
  // and form, M from the reaction's efficiencies; the baths weighted as in the extended PLOG
  void extended_falloff(double cTot) {
    if (!m.i.count("xfo_rxn")) return;
    const auto& xr = m.I("xfo_rxn"); const auto& ki = m.F("xfo_kinf");
    const auto& tp = m.I("xfo_tb_ptr"); const auto& ts = m.I("xfo_tb_sp"); const auto& te = m.F("xfo_tb_eff_m1");
    const auto& bp = m.I("xfo_bath_ptr"); const auto& bs = m.I("xfo_bath_sp"); const auto& lo = m.F("xfo_low");
    const auto& ty = m.I("xfo_type"); const auto& pp = m.I("xfo_par_ptr"); const auto& pa = m.F("xfo_par");
    const double T = T_;
    for (size_t r = 0; r < xr.size(); ++r) {
      const double kInf = ki[3 * r] * std::pow(T, ki[3 * r + 1]) * std::exp(-ki[3 * r + 2] / T);
      double M = cTot;
      for (int q = tp[r]; q < tp[r + 1]; ++q) M += te[q] * c[ts[q]];
      double rest = cTot;
      for (int b = bp[r]; b < bp[r + 1]; ++b) if (bs[b] != -1) rest -= c[bs[b]];
      double kc = 0.;
      for (int b = bp[r]; b < bp[r + 1]; ++b) {
        const double k0 = lo[3 * b] * std::pow(T, lo[3 * b + 1]) * std::exp(-lo[3 * b + 2] / T);
        const double Pr = k0 / kInf * M;
        const double* t = pa.data() + pp[b];
        const int nt = pp[b + 1] - pp[b];
        double F = 1.;
        if (ty[b] == 1) {
          double Fcent = (1. - t[0]) * std::exp(-T / t[1]) + t[0] * std::exp(-T / t[2]);
          if (nt == 4) Fcent += std::exp(-t[3] / T);
          double logFcent = -300.;
          if (Fcent > 1e-300) logFcent = std::log10(Fcent);
          if (Pr > 1.e-32) {
            const double cc = -0.4 - 0.67 * logFcent;
            const double n = 0.75 - 1.27 * logFcent;
            const double e = std::log10(Pr) + cc;
            const double q = e / (n - 0.14 * e);
            F = std::pow(10., logFcent / (1. + q * q));
          } else {
            const double q = 1. / 0.14;
            F = std::pow(10., logFcent / (1. + q * q));
          }
        } else if (ty[b] == 2) {
          const double l = std::log10(Pr);
          const double X = 1. / (1. + l * l);
          F = std::pow(t[0] * std::exp(-t[1] / T) + std::exp(-T / t[2]), X);
          if (nt == 5) F *= t[3] * std::pow(T, t[4]);
        }
        kc += (bs[b] != -1 ? c[bs[b]] : rest) * (kInf * (Pr / (1. + Pr)) * F);
      }
      kc /= cTot;
      kArr[xr[r]] = kc;
      kMod[xr[r]] = kc;
    }
  }

  void reaction_rates(double cTot_given = -1.) {
    double cTot = 0.;
    for (int i = 0; i < NC; ++i) cTot += c[i];
    if (cTot_given >= 0.) cTot = cTot_given;   // ReactionRates(c, cTot) with the caller's cTot
    kinetic_constants();
    extended_plog(cTot);
    const auto& tbr = m.I("tb_rxn"); const auto& tbp = m.I("tb_ptr");
    const auto& tbs = m.I("tb_species"); const auto& tbe = m.F("tb_eff_m1");
    for (size_t sidx = 0; sidx < tbr.size(); ++sidx) {
      double M = cTot;
      for (int q = tbp[sidx]; q < tbp[sidx + 1]; ++q) M += c[tbs[q]] * tbe[q];
      kMod[tbr[sidx]] *= M;
      Mtb[sidx] = M;
    }
    const auto& fr = m.I("fo_rxn"); const auto& fty = m.I("fo_type"); const auto& fsg = m.I("fo_single");
    const auto& fp = m.I("fo_ptr"); const auto& fs = m.I("fo_species"); const auto& fe = m.F("fo_eff_m1");
    const auto& fd = m.F("fo_d"); const auto& fee = m.F("fo_e");
    for (size_t k = 0; k < fr.size(); ++k) {
      double M;
      if (fsg[k] < 0) {
        M = cTot;
        for (int q = fp[k]; q < fp[k + 1]; ++q) M += c[fs[q]] * fe[q];
      } else {
        M = c[fsg[k]] + 1.e-16;
      }
      const int j = fr[k];
      const double Pr = kArr[j] * M / kInf[k];
      const bool cabr = m.i.count("fo_cabr") && m.I("fo_cabr")[k] != 0;
      double wF = 1.;
      if (fty[k] == 1) {
        if (Pr > 1.e-32 || cabr) {   // ChemicallyActivatedBimolecularReactions has no small-Pr branch
          const double nTroe = 0.75 - 1.27 * logFcent[k];
          const double cTroe = -0.4 - 0.67 * logFcent[k];
          const double sTroe = std::log10(Pr) + cTroe;
          const double q = sTroe / (nTroe - 0.14 * sTroe);
          wF = std::pow(10., logFcent[k] / (1. + q * q));
        } else {
          const double q = 1. / 0.14;
          wF = std::pow(10., logFcent[k] / (1. + q * q));
        }
      } else if (fty[k] == 2) {
        const double l = std::log10(Pr);
        const double xSRI = 1. / (1. + l * l);
        wF = std::pow(logFcent[k], xSRI) * fd[k];
        if (fee[k] != 0.) wF *= std::pow(T_, fee[k]);
      }
      // KineticsMap_CHEMKIN::ChemicallyActivatedBimolecularReactions (:1613-1660): correction_cabr = F / (1 + Pr)
      corr[k] = cabr ? (1. / (1. + Pr)) * wF : kInf[k] * (Pr / (1. + Pr)) * wF / kArr[j];
    }
    for (size_t k = 0; k < fr.size(); ++k) kMod[fr[k]] *= corr[k];
    extended_falloff(cTot);

    // StoichiometricMap::ProductOfConcentrations (:512-598): factors in species order, forward orders
    // lambda (FORD or the reactant coefficients)
    const auto& rp = m.I("ford_ptr"); const auto& rs = m.I("ford_species"); const auto& rn = m.F("ford_val");
    const auto& pp = m.I("prod_ptr"); const auto& ps = m.I("prod_species"); const auto& pn = m.F("prod_nu");
    const auto& isrev = m.I("is_reversible");
    for (int j = 0; j < NR; ++j) {
      double pr = 1.;
      for (int q = rp[j]; q < rp[j + 1]; ++q) pr *= conc_factor(rn[q], c[rs[q]]);
      fwd[j] = pr;
      double pv = 1.;
      if (isrev[j]) for (int q = pp[j]; q < pp[j + 1]; ++q) pv *= conc_factor(pn[q], c[ps[q]]);
      rev[j] = pv;
    }
    const auto& rth = m.I("rev_thermo");
    for (size_t k = 0; k < rth.size(); ++k) rev[rth[k]] *= uKeq[k];
    const auto& rex = m.I("rev_explicit");
    for (size_t k = 0; k < rex.size(); ++k) rev[rex[k]] *= kRev[k] / kArr[rex[k]];
    for (int j = 0; j < NR; ++j) net[j] = fwd[j];
    for (int j = 0; j < NR; ++j) if (isrev[j]) net[j] -= rev[j];
    for (int j = 0; j < NR; ++j) net[j] *= kMod[j];
  }
  static double conc_factor(double nu, double c1) {
    if (nu == 1.) return c1;
    if (nu == 2.) return c1 * c1;
    if (nu == 3.) return c1 * c1 * c1;
    if (nu == 0.5) return std::sqrt(c1);
    return std::pow(c1, nu);
  }

  // StoichiometricMap::FormationRatesFromReactionRates (:656-729)
  void formation_rates() {
    const auto& fp = m.I("fr_ptr"); const auto& fr = m.I("fr_rxn"); const auto& fc = m.F("fr_coef");
    for (int i = 0; i < NC; ++i) {
      double rate = 0.;
      for (int q = fp[i]; q < fp[i + 1]; ++q) rate += contrib(fc[q] < 0 ? -fc[q] : fc[q], net[fr[q]]) * (fc[q] < 0 ? -1. : 1.);
      R[i] = rate;
    }
  }

  // DRG-reduced system (BatchReactorHomogeneousConstantPressure.H:253-320): the unknowns are the
  // important species (ascending) and T; the other species keep their values in omega, and the
  // dropped reactions' rates are zeroed before the formation rates.  Constant pressure only.
  const std::vector<int>* drg_species = nullptr;
  const std::vector<int>* drg_dropped = nullptr;
  std::vector<double> omega;

  void equations_drg(const double* y, double* dy) {
    const auto& MW = m.F("mw");
    const std::vector<int>& S = *drg_species;
    const int ni = (int)S.size();
    for (int i = 0; i < ni; ++i) omega[S[i]] = y[i];
    const double T = y[ni];
    double u = 0.;
    for (int i = 0; i < NC; ++i) u += omega[i] / MW[i];
    const double MWmix = 1. / u;
    for (int i = 0; i < NC; ++i) x[i] = MWmix * omega[i];
    for (int i = 0; i < NC; ++i) x[i] = x[i] / MW[i];
    const double cTot = P0 / R_J_KMOL / T;
    for (int i = 0; i < NC; ++i) c[i] = cTot * x[i];
    const double rho = cTot * MWmix;
    P_ = P0;
    h_over_RT(T);
    kin_set_T(T);
    reaction_rates();
    for (int j : *drg_dropped) net[j] = 0.;
    formation_rates();
    for (int i = 0; i < ni; ++i) dy[i] = MW[S[i]] * R[S[i]] / rho;
    dy[ni] = 0.;
    if (energy) {
      cp_over_R(T);
      double cpm = 0.;
      for (int i = 0; i < NC; ++i) cpm += cp[i] * x[i];
      cpm *= R_J_KMOL;
      double d = 0.;
      for (int i = 0; i < NC; ++i) d += R[i] * h[i];
      QR = -d * R_J_KMOL * T;
      const double CpMixMass = cpm / MWmix;
      dy[ni] = QR / (rho * CpMixMass);
    }
  }

  // BatchReactorHomogeneousConstantPressure::Equations (:175-223)
  void equations(const double* y, double* dy) {
    ++n_calls;
    if (drg_species) { equations_drg(y, dy); return; }
    const auto& MW = m.F("mw");
    const double T = y[NC];
    // ThermodynamicsMap_CHEMKIN::MoleFractions_From_MassFractions (:429-434)
    double u = 0.;
    for (int i = 0; i < NC; ++i) u += y[i] / MW[i];
    const double MWmix = 1. / u;
    for (int i = 0; i < NC; ++i) x[i] = MWmix * y[i];
    for (int i = 0; i < NC; ++i) x[i] = x[i] / MW[i];
    // constant volume (BatchReactorHomogeneousConstantVolume.H:148-199): cTot_ = rho0_ / MW_
    const bool cv = rho0 > 0.;
    const double cTot = cv ? rho0 / MWmix : P0 / R_J_KMOL / T;
    for (int i = 0; i < NC; ++i) c[i] = cTot * x[i];
    const double rho = cv ? rho0 : cTot * MWmix;
    P_ = cv ? cTot * R_J_KMOL * T : P0;
    h_over_RT(T);   // species h/RT at T: used by the reaction enthalpies and by QR
    kin_set_T(T);
    reaction_rates();
    formation_rates();
    for (int i = 0; i < NC; ++i) dy[i] = MW[i] * R[i] / rho;
    dy[NC] = 0.;
    if (energy) {
      cp_over_R(T);
      double cpm = 0.;
      for (int i = 0; i < NC; ++i) cpm += cp[i] * x[i];
      cpm *= R_J_KMOL;
      double d = 0.;
      for (int i = 0; i < NC; ++i) d += R[i] * h[i];
      QR = -d * R_J_KMOL * T;
      if (cv) {
        // CvMixMass_ = (CpMixMolar - R) / MW_; dT/dt = (QR_ + R T sum R_i) / (rho0_ CvMixMass_)
        const double CvMixMass = (cpm - R_J_KMOL) / MWmix;
        double sumR = 0.;
        for (int i = 0; i < NC; ++i) sumR += R[i];
        dy[NC] = (QR + R_J_KMOL * T * sumR) / (rho0 * CvMixMass);
      } else {
        const double CpMixMass = cpm / MWmix;
        dy[NC] = QR / (rho * CpMixMass);
      }
    }
  }
};

// ---------------------------------------------------------------------------
// Options and per-cell results
// ---------------------------------------------------------------------------
struct Options {
  double rtol, atol, tmin_chem;
  double y_min_T, y_max_T;
  int max_steps;
  int full_pivoting;
  int energy;
  double alfa2_4, alfa2_5;   // order-selection state carried by the reference's solver object
  int maximum_order;
};

enum { COUNT_STEPS, COUNT_RHS, COUNT_JAC, COUNT_FACT, COUNT_SOLVE, COUNT_ERRFAIL, COUNT_CONVFAIL, COUNT_JAC_RHS, NCOUNT };

// ---------------------------------------------------------------------------
// OdeSMOKE::MultiValueSolver< MethodGear< KernelDense<...> > >
//   math/native-ode-solvers/MultiValueSolver.hpp:40-1328
//   math/native-ode-solvers/MethodGear.hpp:40-568
//   math/native-ode-solvers/KernelDense.hpp:44-245
// ---------------------------------------------------------------------------
class Gear {
 public:
  enum { H_DEC, H_CONST, H_INC };
  enum { O_DEC, O_CONST, O_INC };
  enum { JAC_CHANGE, JAC_MODIFIED, JAC_OK };
  enum { M_TO_FACT, M_FACT };
  enum { CONV_FAIL, CONV_OK };
  static const int MAX_ORDER = 5, MIN_ORDER = 1;
  static const unsigned MAX_ITERATIONS_JACOBIAN = 50, MAX_CONVERGENCE_FAILURE = 50, MAX_ERROR_FAILURE = 50;

  Reactor& sys;
  unsigned ne;
  // method constants (MethodGear.hpp:125-193)
  double r_[MAX_ORDER + 1][MAX_ORDER];
  double Ep_[MAX_ORDER + 1];
  double alfa2_[MAX_ORDER + 1];
  double deltaAlfa1_ = .05, deltaAlfa3_ = .25;
  // state
  std::vector<std::vector<double>> z_, v_;
  std::vector<double> b_, y_, va_, deltab_, f_, vb_, aux_, y0_, oneOverEps_, minv_, maxv_;
  std::vector<double> J_, G_;   // column major n x n
  std::vector<int> piv_;
  double abs_tol_, rel_tol_;
  bool min_c_ = true, max_c_ = true;
  bool full_piv_ = false;
  unsigned maximum_order_ = MAX_ORDER;
  unsigned max_number_steps_ = 500000;
  double max_step_size_ = 1.7976931348623154e+308;
  double min_step_size_ = 0.;
  bool direction_plus_ = true;
  // MultiValueSolver scalars
  double t_, t0_, tOut_, tInMeshPoint_, tStabilize_;
  double hPreviousStep_, hNordsieck_, hScaleMax_, first_step_size_;
  bool fixedOrderMin_;
  unsigned iterOfConstStepsForLargeFactorizationTime_, iterConstSteps_, iterMinimumOrder_;
  double cpuTimeEquationSystem_ = 0., cpuTimeToFactorize_ = 0.;
  // MethodGear scalars
  unsigned p_, iterOrder_, orderInNextStep_, maxConvergenceIterations_, maxIterationsJacobian_;
  int odeHStatus_, odeOrderStatus_, status_, factorizationStatus_, jacobianStatus_, convergenceStatus_;
  double h_, hNextStep_, hScale_;
  unsigned numberOfSteps_, iterConvergence_, iterConvergenceRate_, iterConvergenceFailure_, iterErrorFailure_;
  unsigned numberOfConvergenceFailuresForOrderMax_;
  unsigned stepOfLastJacobian_ = 0, stepOfLastFactorization_ = 0;
  long long cnt_[NCOUNT];

  explicit Gear(Reactor& s, unsigned n) : sys(s), ne(n) {
    // MethodGear::MemoryAllocationMethod (:125-193)
    for (int i = 0; i <= MAX_ORDER; ++i) alfa2_[i] = .8;
    for (int j = 0; j <= MAX_ORDER; ++j) Ep_[j] = (double)factorial(j);
    for (int i = 0; i <= MAX_ORDER; ++i) for (int j = 0; j < MAX_ORDER; ++j) r_[i][j] = 0.;
    r_[0][0] = 1.; r_[1][0] = 1.;
    for (int j = 2; j <= MAX_ORDER; ++j) {
      r_[0][j - 1] = (double)factorial(j);
      for (int i = 2; i <= j; ++i) r_[i - 1][j - 1] = double(j) * r_[i - 1][j - 2] + r_[i - 2][j - 2];
      r_[j][j - 1] = 1.;
    }
    double sum = 1.;
    for (int j = 2; j <= MAX_ORDER; ++j) {
      sum += 1. / double(j);
      for (int i = 1; i <= j + 1; ++i) r_[i - 1][j - 1] /= (factorial(j) * sum);
    }
    z_.assign(MAX_ORDER + 3, std::vector<double>(n, 0.));
    v_.assign(MAX_ORDER + 3, std::vector<double>(n, 0.));
    b_.assign(n, 0.); y_.assign(n, 0.); va_.assign(n, 0.); deltab_.assign(n, 0.); f_.assign(n, 0.);
    vb_.assign(n, 0.); aux_.assign(n, 0.); y0_.assign(n, 0.); oneOverEps_.assign(n, 0.);
    minv_.assign(n, 0.); maxv_.assign(n, 0.);
    J_.assign((size_t)n * n, 0.); G_.assign((size_t)n * n, 0.); piv_.assign(n, 0);
  }
  static unsigned factorial(unsigned n) { return n == 0 ? 1 : n * factorial(n - 1); }

  void equations(const std::vector<double>& y, std::vector<double>& dy) { sys.equations(y.data(), dy.data()); ++cnt_[COUNT_RHS]; }

  static double error_control(const std::vector<double>& w, const std::vector<double>& e) {
    // math/OpenSMOKEUtilities.hpp:689-701
    double sum = 0.;
    for (size_t i = 0; i < w.size(); ++i) { const double c = w[i] * e[i]; sum += c * c; }
    return std::sqrt(sum / double(w.size()));
  }

  // MultiValueSolver::SetInitialConditions (:367-407) with MethodGear::ResetMethod (:79-123)
  // and MultiValueSolver::Reset (:107-134)
  void set_initial_conditions(double t0, const double* y0) {
    tOut_ = t_ = t0_ = tInMeshPoint_ = tStabilize_ = t0;
    full_piv_ = false;
    p_ = 1; iterOrder_ = 0; orderInNextStep_ = 1; maxConvergenceIterations_ = 4;
    maxIterationsJacobian_ = 20 + 5 * (ne - 3);
    if (maxIterationsJacobian_ > MAX_ITERATIONS_JACOBIAN && ne < 80) maxIterationsJacobian_ = MAX_ITERATIONS_JACOBIAN;
    odeHStatus_ = H_CONST; odeOrderStatus_ = O_CONST; status_ = 1;
    factorizationStatus_ = M_TO_FACT; jacobianStatus_ = JAC_CHANGE; convergenceStatus_ = CONV_OK;
    h_ = 0.; min_step_size_ = 0.; hNextStep_ = 0.; hScale_ = 0.;
    numberOfSteps_ = 0; numberOfConvergenceFailuresForOrderMax_ = 0;
    iterConvergence_ = 0; iterConvergenceRate_ = 0; iterConvergenceFailure_ = 0; iterErrorFailure_ = 0;
    for (unsigned i = 0; i < ne; ++i) y0_[i] = y0[i];
    hPreviousStep_ = 0.; hNordsieck_ = 0.; hScaleMax_ = 1000.;
    fixedOrderMin_ = false;
    iterOfConstStepsForLargeFactorizationTime_ = 0; iterConstSteps_ = 0; iterMinimumOrder_ = 0;
    for (int k = 0; k < NCOUNT; ++k) cnt_[k] = 0;
    equations(y0_, f_);
  }

  void check_constraints(std::vector<double>& y) {   // MethodGear::CheckConstraints (:518-536)
    if (min_c_) for (unsigned i = 0; i < ne; ++i) if (y[i] < minv_[i]) y[i] = minv_[i];
    if (max_c_) for (unsigned i = 0; i < ne; ++i) if (y[i] > maxv_[i]) y[i] = maxv_[i];
  }
  unsigned check_illegal(const std::vector<double>& y) {  // MethodGear::CheckIllegalConstraints (:538-568)
    unsigned n = 0;
    if (min_c_) for (unsigned i = 0; i < ne; ++i) if (y[i] < minv_[i]) ++n;
    if (max_c_) for (unsigned i = 0; i < ne; ++i) if (y[i] > maxv_[i]) ++n;
    return n;
  }

  void one_over_epsilon(const std::vector<double>& w) {   // MultiValueSolver.hpp:619-645
    for (unsigned i = 0; i < ne; ++i) oneOverEps_[i] = abs_tol_ + rel_tol_ * std::fabs(w[i]);
    for (unsigned i = 0; i < ne; ++i) oneOverEps_[i] = 1. / oneOverEps_[i];
  }

  double initial_step() {   // MultiValueSolver.hpp:648-685
    double lo, hi;
    if (t0_ != 0.) { lo = 100. * MACH_EPS_DOUBLE * std::fabs(t0_); hi = std::fabs(t0_); }
    else { lo = MACH_EPS_DOUBLE; hi = 1.e-4; }
    one_over_epsilon(y0_);
    double h0 = 0.5 / (error_control(f_, oneOverEps_) + MACH_EPS_FLOAT);
    if (h0 < lo) h0 = lo;
    if (h0 > hi) h0 = hi;
    h0 *= std::fabs(tOut_ - t0_) / (tOut_ - t0_);
    return h0;
  }

  void interpolation() {   // MultiValueSolver.hpp:687-706
    const double hp = (tOut_ - t_) / hNordsieck_;
    double hr = 1.;
    y_ = z_[0];
    if (hp == 0.) return;
    for (unsigned i = 1; i <= p_; ++i) {
      hr *= hp;
      for (unsigned k = 0; k < ne; ++k) va_[k] = z_[i][k] * hr;
      for (unsigned k = 0; k < ne; ++k) y_[k] += va_[k];
    }
    check_constraints(y_);
  }

  // KernelDense::NumericalJacobian (:111-193), constrained branch taken when max constraints are on
  void numerical_jacobian(std::vector<double>& y, const std::vector<double>& f, double h, const std::vector<double>& e) {
    const double ZERO_DER = std::sqrt(TINY_FLOAT);
    const double ETA2 = std::sqrt(MACH_EPS_DOUBLE);
    const double BETA = 1.e+3 * MACH_EPS_DOUBLE;
    double hf = BETA * std::fabs(h) * error_control(f, e) * double(ne);
    if (hf < 1.e-10) hf = 1.;
    for (unsigned j = 0; j < ne; ++j) {
      const double yh = y[j];
      double hJ;
      if (!max_c_) {
        hJ = ETA2 * std::fabs(std::max(yh, 1. / e[j]));
        const double hJf = hf / e[j];
        hJ = std::max(hJ, hJf);
        hJ = std::max(hJ, ZERO_DER);
        hJ = std::min(hJ, 0.001 + 0.001 * std::fabs(yh));
      } else {
        const double a = std::fabs(yh), b = std::fabs(1. / e[j]);
        hJ = ETA2 * (a > b ? a : b);
        const double hJf = hf / e[j];
        hJ = std::max(hJ, hJf);
        hJ = std::max(hJ, ZERO_DER);
        if (yh + hJ > maxv_[j]) hJ = -hJ;
      }
      y[j] += hJ;
      sys.equations(y.data(), aux_.data());
      ++cnt_[COUNT_JAC_RHS];
      y[j] = yh;
      for (unsigned i = 0; i < ne; ++i) aux_[i] -= f[i];
      const double hInv = 1. / hJ;
      for (unsigned i = 0; i < ne; ++i) J_[(size_t)j * ne + i] = hInv * aux_[i];
    }
  }

  // KernelDense::BuildAndFactorizeMatrixG (:195-220): G = I - hr0 J, partial-pivot LU
  // (Eigen::PartialPivLU picks the row of largest magnitude in the column).
  void build_and_factorize(double hr0) {
    for (size_t q = 0; q < G_.size(); ++q) G_[q] = J_[q];
    for (size_t q = 0; q < G_.size(); ++q) G_[q] *= -hr0;
    for (unsigned i = 0; i < ne; ++i) G_[(size_t)i * ne + i] += 1.;
    const unsigned n = ne;
    for (unsigned k = 0; k < n; ++k) {
      unsigned pr = k; double best = std::fabs(G_[(size_t)k * n + k]);
      for (unsigned i = k + 1; i < n; ++i) { const double a = std::fabs(G_[(size_t)k * n + i]); if (a > best) { best = a; pr = i; } }
      piv_[k] = (int)pr;
      if (pr != k) for (unsigned j = 0; j < n; ++j) std::swap(G_[(size_t)j * n + k], G_[(size_t)j * n + pr]);
      const double d = G_[(size_t)k * n + k];
      if (d != 0.) for (unsigned i = k + 1; i < n; ++i) G_[(size_t)k * n + i] /= d;
      for (unsigned j = k + 1; j < n; ++j) {
        const double ukj = G_[(size_t)j * n + k];
        for (unsigned i = k + 1; i < n; ++i) G_[(size_t)j * n + i] -= G_[(size_t)k * n + i] * ukj;
      }
    }
    ++cnt_[COUNT_FACT];
  }

  void solve_linear_system(std::vector<double>& db) {   // KernelDense::SolveLinearSystem (:222-245)
    const unsigned n = ne;
    for (unsigned k = 0; k < n; ++k) if (piv_[k] != (int)k) std::swap(db[k], db[piv_[k]]);
    for (unsigned j = 0; j < n; ++j) { const double v = db[j]; for (unsigned i = j + 1; i < n; ++i) db[i] -= G_[(size_t)j * n + i] * v; }
    for (int j = (int)n - 1; j >= 0; --j) {
      db[j] /= G_[(size_t)j * n + j];
      const double v = db[j];
      for (int i = 0; i < j; ++i) db[i] -= G_[(size_t)j * n + i] * v;
    }
    ++cnt_[COUNT_SOLVE];
  }

  void jacobian_times_vector(const std::vector<double>& vin, std::vector<double>& vout) {   // KernelDense.hpp:90-94
    for (unsigned i = 0; i < ne; ++i) {
      double s = 0.;
      for (unsigned j = 0; j < ne; ++j) s += J_[(size_t)j * ne + i] * vin[j];
      vout[i] = s;
    }
  }

  // MethodGear::FindCorrection (:195-341)
  unsigned find_correction(double t) {
    vb_ = v_[0];
    check_constraints(vb_);
    equations(vb_, f_);
    if (numberOfSteps_ >= stepOfLastJacobian_ + maxIterationsJacobian_) jacobianStatus_ = JAC_CHANGE;
    if (jacobianStatus_ == JAC_CHANGE) {
      stepOfLastJacobian_ = numberOfSteps_;
      jacobianStatus_ = JAC_MODIFIED;
      numerical_jacobian(vb_, f_, h_, oneOverEps_);
      ++cnt_[COUNT_JAC];
      factorizationStatus_ = M_TO_FACT;
    }
    const double hr0 = h_ * r_[0][p_ - 1];
    if (factorizationStatus_ == M_FACT && iterOrder_ == 0) factorizationStatus_ = M_TO_FACT;
    if (factorizationStatus_ == M_TO_FACT) {
      stepOfLastFactorization_ = numberOfSteps_;
      build_and_factorize(hr0);
      factorizationStatus_ = M_FACT;
    }
    for (unsigned i = 0; i < ne; ++i) deltab_[i] = f_[i] * h_;
    for (unsigned i = 0; i < ne; ++i) deltab_[i] -= v_[1][i];
    solve_linear_system(deltab_);
    b_ = deltab_;
    double oldCC = 0.;
    for (unsigned k = 1; k <= maxConvergenceIterations_; ++k) {
      const double cc = r_[0][p_ - 1] * error_control(deltab_, oneOverEps_);
      if (cc < 1.) { convergenceStatus_ = CONV_OK; return k; }
      if (k > 1 && cc > 2. * oldCC) { convergenceStatus_ = CONV_FAIL; return k; }
      oldCC = cc;
      for (unsigned i = 0; i < ne; ++i) va_[i] = b_[i] * r_[0][p_ - 1];
      for (unsigned i = 0; i < ne; ++i) va_[i] += v_[0][i];
      if (min_c_) for (unsigned j = 0; j < ne; ++j) if (va_[j] < minv_[j]) { va_[j] = minv_[j]; b_[j] = (minv_[j] - z_[0][j]) / r_[0][p_ - 1]; }
      if (max_c_) for (unsigned j = 0; j < ne; ++j) if (va_[j] > maxv_[j]) { va_[j] = maxv_[j]; b_[j] = (maxv_[j] - z_[0][j]) / r_[0][p_ - 1]; }
      equations(va_, f_);
      for (unsigned i = 0; i < ne; ++i) deltab_[i] = f_[i] * h_;
      for (unsigned i = 0; i < ne; ++i) deltab_[i] -= v_[1][i];
      for (unsigned i = 0; i < ne; ++i) deltab_[i] -= b_[i];
      solve_linear_system(deltab_);
      for (unsigned i = 0; i < ne; ++i) b_[i] += deltab_[i];
    }
    convergenceStatus_ = CONV_FAIL;
    return maxConvergenceIterations_;
  }

  // MethodGear::WhatToDoInCaseOfConvergenceFailure (:343-423)
  void convergence_failure_recovery() {
    hScale_ = 0.25;
    if (numberOfSteps_ < 10) hScale_ = 0.1;
    hScale_ = std::max(hScale_, min_step_size_ / std::fabs(h_));
    odeHStatus_ = H_DEC;
    if (p_ > (unsigned)MIN_ORDER) { p_ -= 1; odeOrderStatus_ = O_DEC; }
    alfa2_[4] -= 0.01;
    alfa2_[5] -= 0.02;
    if (alfa2_[4] < 0.) { alfa2_[4] = 0.; maximum_order_ = 3; if (p_ > 3) { p_ = 3; odeOrderStatus_ = O_DEC; } }
    if (alfa2_[5] < 0.) { alfa2_[5] = 0.; maximum_order_ = 4; if (p_ > 4) { p_ = 4; odeOrderStatus_ = O_DEC; } }
    if (numberOfSteps_ > 5) {
      numberOfConvergenceFailuresForOrderMax_++;
      if (numberOfConvergenceFailuresForOrderMax_ % 5 == 0) {
        if (p_ != (unsigned)MIN_ORDER) { p_ = MIN_ORDER; odeOrderStatus_ = O_DEC; }
      }
      if (numberOfConvergenceFailuresForOrderMax_ % 10 == 0 && tStabilize_ != tInMeshPoint_) {
        equations(z_[0], va_);
        for (unsigned i = 0; i < ne; ++i) z_[1][i] = va_[i] * h_;
        tStabilize_ = tInMeshPoint_;
      }
    }
    if (numberOfSteps_ > stepOfLastJacobian_ + MAX_ITERATIONS_JACOBIAN / 10) jacobianStatus_ = JAC_CHANGE;
    if (numberOfSteps_ != stepOfLastJacobian_ && iterConvergenceFailure_ == MAX_CONVERGENCE_FAILURE) jacobianStatus_ = JAC_CHANGE;
    hNextStep_ *= hScale_;
  }

  // MethodGear::ConvergenceRate (:425-516)
  void convergence_rate() {
    if (iterErrorFailure_ > 0 || iterConvergenceFailure_ > 0) iterConvergenceRate_ = 0;
    if (iterConvergence_ <= 1) return;
    for (unsigned i = 0; i < ne; ++i) vb_[i] = v_[0][i] - z_[0][i];
    jacobian_times_vector(vb_, va_);
    for (unsigned i = 0; i < ne; ++i) va_[i] *= h_;
    for (unsigned i = 0; i < ne; ++i) va_[i] += z_[1][i];
    for (unsigned i = 0; i < ne; ++i) va_[i] = v_[1][i] - va_[i];
    double normd = 0., normf = 0.;
    for (unsigned i = 0; i < ne; ++i) normd += std::fabs(va_[i]);
    for (unsigned i = 0; i < ne; ++i) normf += std::fabs(v_[1][i]);
    if (normd > 3. * normf + .1 && iterConvergence_ > 2) {
      if (numberOfSteps_ > stepOfLastJacobian_ + MAX_ITERATIONS_JACOBIAN / 10) jacobianStatus_ = JAC_CHANGE;
      hScale_ = 0.5; odeHStatus_ = H_DEC; hNextStep_ = h_ * hScale_;
      if (p_ > 1) { orderInNextStep_ = p_ - 1; odeOrderStatus_ = O_DEC; }
      iterConvergenceRate_ = 0; iterConvergenceFailure_ = 1;
      return;
    }
    if (normd > normf + 0.1) {
      iterConvergenceRate_++;
      if (iterConvergenceRate_ >= 5) {
        hScale_ = 0.8; odeHStatus_ = H_DEC; hNextStep_ = h_ * hScale_;
        iterConvergenceRate_ = 0; iterConvergenceFailure_ = 1;
      }
      if (numberOfSteps_ > stepOfLastJacobian_ + MAX_ITERATIONS_JACOBIAN / 10 && iterConvergence_ > 2) {
        jacobianStatus_ = JAC_CHANGE;
        iterConvergenceRate_ = 0; iterConvergenceFailure_ = 1;
      }
    }
  }

  // MultiValueSolver::MultiValueStep (:1212-1328)
  void multi_value_step() {
    for (unsigned i = 0; i <= p_; ++i) v_[i] = z_[i];
    for (int i = 0; i < int(p_); ++i)
      for (int j = int(p_ - 1); j >= i; --j)
        for (unsigned k = 0; k < ne; ++k) v_[j][k] += v_[j + 1][k];
    if (min_c_) for (unsigned j = 0; j < ne; ++j) if (v_[0][j] < minv_[j]) {
      if (std::fabs(v_[0][j] - minv_[j]) * oneOverEps_[j] < double(ne)) {
        v_[0][j] = minv_[j]; v_[1][j] = minv_[j] - z_[0][j];
        for (unsigned i = 2; i <= p_; ++i) v_[i][j] = 0.;
      }
    }
    if (max_c_) for (unsigned j = 0; j < ne; ++j) if (v_[0][j] > maxv_[j]) {
      if (std::fabs(v_[0][j] - maxv_[j]) * oneOverEps_[j] < double(ne)) {
        v_[0][j] = maxv_[j]; v_[1][j] = maxv_[j] - z_[0][j];
        for (unsigned i = 2; i <= p_; ++i) v_[i][j] = 0.;
      }
    }
    iterConvergence_ = find_correction(t_);
    if (convergenceStatus_ == CONV_FAIL) return;
    const double r0 = r_[0][p_ - 1];
    for (unsigned i = 0; i < ne; ++i) va_[i] = b_[i] * r0;
    if (min_c_) for (unsigned j = 0; j < ne; ++j) if (v_[0][j] + va_[j] < minv_[j]) {
      b_[j] = minv_[j] - z_[0][j] - v_[1][j];
      v_[0][j] = minv_[j] - va_[j];
      if (v_[0][j] < minv_[j]) v_[0][j] = minv_[j];
    }
    if (max_c_) for (unsigned j = 0; j < ne; ++j) if (v_[0][j] + va_[j] > maxv_[j]) {
      b_[j] = maxv_[j] - z_[0][j] - v_[1][j];
      v_[0][j] = maxv_[j] - va_[j];
      if (v_[0][j] > maxv_[j]) v_[0][j] = maxv_[j];
    }
    for (unsigned k = 0; k < ne; ++k) v_[0][k] += va_[k];
    for (unsigned k = 0; k < ne; ++k) v_[1][k] += b_[k];
    for (unsigned i = 2; i <= p_; ++i) {
      const double ri = r_[i][p_ - 1];
      for (unsigned k = 0; k < ne; ++k) va_[k] = b_[k] * ri;
      for (unsigned k = 0; k < ne; ++k) v_[i][k] += va_[k];
    }
    for (unsigned k = 0; k < ne; ++k) va_[k] = v_[p_][k] - z_[p_][k];
    for (unsigned k = 0; k < ne; ++k) v_[p_ + 1][k] = va_[k] / (double(p_) + 1.);
    if (iterOrder_ >= p_) {
      for (unsigned k = 0; k < ne; ++k) va_[k] = v_[p_ + 1][k] - z_[p_ + 1][k];
      for (unsigned k = 0; k < ne; ++k) v_[p_ + 2][k] = va_[k] / (double(p_) + 2.);
    }
  }

  // MultiValueSolver::NewOrderNewH (:1042-1210); the CPU-time heuristics are
  // always false because cpuTimeToFactorize_ stays 0 (MultiValueSolver.hpp:133).
  void new_order_new_h() {
    double hMinus = 0., hCur = 0., hPlus = 0., alfa1 = 0., alfa3 = 0.;
    if (p_ > (unsigned)MIN_ORDER && odeOrderStatus_ != O_INC) {
      hMinus = Ep_[p_ - 1] * error_control(v_[p_], oneOverEps_) + MACH_EPS_FLOAT;
      hMinus = 1. / hMinus;
      alfa1 = alfa2_[p_ - 1] - deltaAlfa1_;
      hMinus = alfa1 * std::pow(hMinus, 1. / double(p_));
    }
    {
      hCur = Ep_[p_] * error_control(v_[p_ + 1], oneOverEps_) + MACH_EPS_FLOAT;
      hCur = 1. / hCur;
      hCur = alfa2_[p_] * std::pow(hCur, 1. / double(p_ + 1));
    }
    if (p_ < maximum_order_ && odeOrderStatus_ != O_DEC) {
      hPlus = Ep_[p_ + 1] * error_control(v_[p_ + 2], oneOverEps_) + MACH_EPS_FLOAT;
      hPlus = 1. / hPlus;
      alfa3 = alfa2_[p_ + 1] - deltaAlfa3_;
      hPlus = alfa3 * std::pow(hPlus, 1. / double(p_ + 2));
    }
    if (hMinus > hCur && hMinus > hPlus) {
      hScale_ = (.75 / alfa1) * hMinus; orderInNextStep_ = p_ - 1; odeOrderStatus_ = O_DEC;
    } else if (hCur > hMinus && hCur > hPlus) {
      hScale_ = (.75 / alfa2_[p_]) * hCur; orderInNextStep_ = p_; odeOrderStatus_ = O_CONST;
    } else {
      hScale_ = (.75 / alfa3) * hPlus; orderInNextStep_ = p_ + 1; odeOrderStatus_ = O_INC;
    }
    if (fixedOrderMin_) {
      iterMinimumOrder_++;
      if (iterMinimumOrder_ < 2000) {
        hScale_ = (.75 / alfa2_[p_]) * hCur; orderInNextStep_ = p_; odeOrderStatus_ = O_CONST;
      } else fixedOrderMin_ = false;
    }
    {
      double scl = 1.2;
      if (hScale_ < scl) {
        iterOfConstStepsForLargeFactorizationTime_ = 0;
        iterConstSteps_++;
        hScale_ = 1.; odeHStatus_ = H_CONST; orderInNextStep_ = p_; odeOrderStatus_ = O_CONST; hNextStep_ = h_;
      } else {
        iterConstSteps_ = 0;
        hScale_ = std::min(hScale_, hScaleMax_);
        odeHStatus_ = H_INC;
        hNextStep_ = h_ * hScale_;
        if (hNextStep_ > max_step_size_) hNextStep_ = max_step_size_;
      }
    }
    if (iterConstSteps_ > 500 || (numberOfSteps_ % 1000 == 0 && numberOfSteps_ != 0 &&
                                  (std::fabs(h_) < 1.e-7 || std::fabs(h_) < 1.e-5 * t_))) {
      if (p_ > (unsigned)MIN_ORDER) {
        fixedOrderMin_ = true; iterMinimumOrder_ = 0;
        orderInNextStep_ = MIN_ORDER; odeOrderStatus_ = O_DEC;
        hScale_ = 0.5; hNextStep_ = h_ * hScale_; odeHStatus_ = H_DEC;
      }
    }
  }

  // MultiValueSolver::DriverStep (:753-1040)
  void driver_step() {
    iterConvergenceFailure_ = 0; iterErrorFailure_ = 0; convergenceStatus_ = CONV_OK;
    if (odeOrderStatus_ != O_CONST || odeHStatus_ != H_CONST) iterOrder_ = 0;
    p_ = orderInNextStep_;
    odeOrderStatus_ = O_CONST;
    hScaleMax_ = 2.;
    if (numberOfSteps_ < 10) hScaleMax_ = 1000.;
    else if (numberOfSteps_ > 10 && numberOfSteps_ < 20) hScaleMax_ = 10.;
    while (true) {
      if (odeHStatus_ != H_CONST) {
        hScale_ = hNextStep_ / hNordsieck_;
        double hr = 1.;
        for (unsigned i = 1; i <= p_; ++i) { hr *= hScale_; for (unsigned k = 0; k < ne; ++k) z_[i][k] *= hr; }
        check_constraints(z_[0]);
        iterOrder_ = 0;
        odeHStatus_ = H_CONST;
      }
      h_ = hNextStep_;
      hNordsieck_ = hNextStep_;
      if (std::fabs(h_) < MACH_EPS_FLOAT * min_step_size_) { status_ = -6; return; }
      t_ = tInMeshPoint_ + h_;
      if (t_ == tInMeshPoint_) { status_ = -6; return; }
      multi_value_step();
      if (convergenceStatus_ == CONV_FAIL) {
        iterConvergenceFailure_++;
        ++cnt_[COUNT_CONVFAIL];
        if (iterConvergenceFailure_ >= MAX_CONVERGENCE_FAILURE) { status_ = -5; return; }
        if (std::fabs(h_ - min_step_size_) <= MACH_EPS_DOUBLE * std::fabs(min_step_size_)) { status_ = -6; return; }
        convergence_failure_recovery();
      } else {
        double hCur = Ep_[p_] * error_control(v_[p_ + 1], oneOverEps_);
        if (hCur > 1.) {
          iterErrorFailure_++;
          ++cnt_[COUNT_ERRFAIL];
          if (iterErrorFailure_ >= MAX_ERROR_FAILURE) { status_ = -4; return; }
          if (std::fabs(h_ - min_step_size_) <= MACH_EPS_DOUBLE * std::fabs(min_step_size_)) { status_ = -6; return; }
          hScaleMax_ = 1.;
          hCur = 0.8 * std::pow(1. / hCur, 1. / double(p_ + 1));
          hScale_ = hCur;
          if (p_ > (unsigned)MIN_ORDER) {
            double hMinus = Ep_[p_ - 1] * error_control(v_[p_], oneOverEps_);
            hMinus = 1. / (hMinus + MACH_EPS_FLOAT);
            hMinus = 0.8 * std::pow(hMinus, 1. / double(p_));
            if (hMinus > hCur) { hScale_ = hMinus; p_ -= 1; odeOrderStatus_ = O_DEC; }
          }
          hScale_ = std::min(hScale_, 0.5);
          hScale_ = std::max(hScale_, min_step_size_ / std::fabs(h_));
          hScale_ = std::max(hScale_, 1.e-3);
          if (p_ == 1 && hScale_ < 0.1 && numberOfSteps_ > 10 && tInMeshPoint_ != tStabilize_) {
            equations(z_[0], va_);
            for (unsigned i = 0; i < ne; ++i) z_[1][i] = va_[i] * h_;
            tStabilize_ = tInMeshPoint_;
          }
          odeHStatus_ = H_DEC;
          hNextStep_ *= hScale_;
        } else {
          hNordsieck_ = h_; hPreviousStep_ = h_; hNextStep_ = h_;
          orderInNextStep_ = p_; odeOrderStatus_ = O_CONST; odeHStatus_ = H_CONST;
          convergence_rate();
          if (iterErrorFailure_ > 0 || iterConvergenceFailure_ > 0) { iterErrorFailure_ = 0; iterConvergenceFailure_ = 0; }
          else { iterOrder_++; if (iterOrder_ > p_ + 1) new_order_new_h(); }
          for (unsigned i = 0; i <= p_ + 2; ++i) z_[i] = v_[i];
          check_constraints(z_[0]);
          break;
        }
      }
    }
  }

  // MultiValueSolver::Solve (:423-617), first call after SetInitialConditions.
  // Returns the status; on failure y_ holds the last accepted state (the
  // reference would hand back stale data here, MultiValueSolver.hpp:567-574).
  int solve(double tOut) {
    tOut_ = tOut;
    if (t0_ > tOut_) direction_plus_ = false;
    if (check_illegal(y0_) != 0) { status_ = -9; y_ = y0_; return status_; }
    first_step_size_ = initial_step();
    z_[0] = y0_;
    for (unsigned i = 0; i < ne; ++i) z_[1][i] = f_[i] * first_step_size_;
    hPreviousStep_ = first_step_size_; hNordsieck_ = first_step_size_; hNextStep_ = first_step_size_;
    status_ = 2;
    for (unsigned k = 1; k <= max_number_steps_; ++k) {
      one_over_epsilon(z_[0]);
      const double tolSafe = MACH_EPS_DOUBLE * error_control(z_[0], oneOverEps_);
      if (tolSafe > 1.) { status_ = -2; y_ = z_[0]; return status_; }
      tInMeshPoint_ = t_;
      driver_step();
      if (status_ <= 0) { t_ = tInMeshPoint_; y_ = z_[0]; return status_; }
      numberOfSteps_++;
      ++cnt_[COUNT_STEPS];
      if (tOut_ == t_) { y_ = z_[0]; return status_; }
      if ((direction_plus_ && tOut_ < t_) || (!direction_plus_ && tOut_ > t_)) {
        interpolation();
        equations(y_, va_);   // printResults_ == true: sets the reactor's QR at tOut (:605-609)
        return status_;
      }
    }
    status_ = -1;
    y_ = z_[0];
    return status_;
  }
};

// ---------------------------------------------------------------------------
// Directed relation graph of one state (solvers/laminarSMOKE/unsteady/DRG.hpp)
// ---------------------------------------------------------------------------
struct Drg {
  const Mech& m;
  int NS, NR;
  // net coefficients nu(k, j) = products - reactants of reaction k, the non-zero ones by species
  // (the constructor's nu_ and delta_, DRG.hpp:45-110)
  std::vector<std::vector<std::pair<int, double>>> nu;
  std::vector<double> den, num;

  explicit Drg(const Mech& mech) : m(mech), NS(mech.nc), NR(mech.nr) {
    const auto& rp = m.I("reac_ptr"); const auto& rs = m.I("reac_species"); const auto& rn = m.F("reac_nu");
    const auto& pp = m.I("prod_ptr"); const auto& ps = m.I("prod_species"); const auto& pn = m.F("prod_nu");
    nu.resize(NR);
    std::vector<double> row(NS);
    for (int k = 0; k < NR; ++k) {
      std::fill(row.begin(), row.end(), 0.);
      for (int q = pp[k]; q < pp[k + 1]; ++q) row[ps[q]] += pn[q];
      for (int q = rp[k]; q < rp[k + 1]; ++q) row[rs[q]] -= rn[q];
      for (int j = 0; j < NS; ++j) if (row[j] != 0.) nu[k].push_back({j, row[j]});
    }
    den.resize(NS); num.resize(NS);
  }

  // Analysis = PairWiseErrorMatrix + ParsePairWiseErrorMatrix (DRG.hpp:150-273) at (T, P, c):
  // r_ij = sum_k |nu_ki r_k| over the reactions with both i and j / (1e-64 + sum_k |nu_ki r_k|),
  // breadth-first from the key species through r_qj > eps; a reaction is dropped when one of its
  // species is not reached.  The rows r_q. are formed when q leaves the queue.
  void analysis(Reactor& R, double T, double P, const double* c, double eps, const std::vector<int>& key,
                std::vector<int>& important, std::vector<int>& dropped) {
    for (int i = 0; i < NS; ++i) R.c[i] = c[i];
    R.P_ = P;
    R.h_over_RT(T);
    R.kin_set_T(T);
    R.reaction_rates();
    const std::vector<double>& r = R.net;
    std::fill(den.begin(), den.end(), 0.);
    for (int k = 0; k < NR; ++k)
      for (const auto& e : nu[k]) den[e.first] += std::fabs(e.second * r[k]);
    std::vector<char> imp(NS, 0);
    std::vector<int> Q;
    size_t head = 0;
    for (int s : key) { Q.push_back(s); imp[s] = 1; }
    while (head < Q.size()) {
      const int q = Q[head];
      std::fill(num.begin(), num.end(), 0.);
      for (int k = 0; k < NR; ++k) {
        double nq = 0.;
        bool has = false;
        for (const auto& e : nu[k]) if (e.first == q) { nq = e.second; has = true; break; }
        if (!has) continue;
        for (const auto& e : nu[k]) num[e.first] += std::fabs(nq * r[k]);
      }
      for (int k = 0; k < NS; ++k)
        if (!imp[k] && num[k] / (1.e-64 + den[q]) > eps) { imp[k] = 1; Q.push_back(k); }
      ++head;
    }
    important.clear();
    for (int k = 0; k < NS; ++k) if (imp[k]) important.push_back(k);
    dropped.clear();
    for (int k = 0; k < NR; ++k) {
      bool keep = true;
      for (const auto& e : nu[k]) if (!imp[e.first]) keep = false;
      if (!keep) dropped.push_back(k);
    }
  }
};

}  // namespace orc

// ---------------------------------------------------------------------------
// C interface used by the tests and by bench.py's CPU baseline.
// ---------------------------------------------------------------------------
extern "C" {

struct orc_options {
  double rtol, atol, tmin_chem, y_min_T, y_max_T;
  int max_steps, full_pivoting, energy;
  double alfa2_4, alfa2_5;
  int maximum_order;
  int sequential_state;   // 1: carry alfa2/maximum_order across cells like one solver object per rank
};

void* orc_mech_load(const void* blob, size_t n) {
  try { return orc::load_blob((const unsigned char*)blob, n); } catch (...) { return nullptr; }
}
void orc_mech_free(void* m) { delete (orc::Mech*)m; }

// One right-hand side evaluation: y = [Y_1..Y_NC, T] -> dy, and the heat release.
int orc_rhs(void* mech, double P, const double* y, double* dy, double* qr) {
  const orc::Mech& m = *(const orc::Mech*)mech;
  orc::Reactor r(m);
  r.P0 = P;
  r.equations(y, dy);
  if (qr) *qr = r.QR;
  return 0;
}

// Finite-difference Jacobian exactly as the solver builds it (for tests).
int orc_fd_jacobian(void* mech, double P, const double* y, double h, double rtol, double atol,
                    double y_max_T, double* J_colmajor) {
  const orc::Mech& m = *(const orc::Mech*)mech;
  orc::Reactor r(m);
  r.P0 = P;
  const unsigned n = m.nc + 1;
  orc::Gear g(r, n);
  for (unsigned i = 0; i < n; ++i) { g.minv_[i] = 0.; g.maxv_[i] = 1.; }
  g.minv_[n - 1] = 200.; g.maxv_[n - 1] = y_max_T;
  g.abs_tol_ = atol; g.rel_tol_ = rtol;
  std::vector<double> yy(y, y + n), f(n);
  r.equations(yy.data(), f.data());
  g.one_over_epsilon(yy);
  g.numerical_jacobian(yy, f, h, g.oneOverEps_);
  std::memcpy(J_colmajor, g.J_.data(), sizeof(double) * n * n);
  return 0;
}

// Batched reaction step, cell-major state Y[ncells][NC] (in/out), T[ncells] (in/out).
// solvers/laminarSMOKE/unsteady/chemistry_DI.H:76-331 (OpenSMOKE native branch)
// and solvers/laminarSMOKE/utilities.H:153-200 (normalizeMassFractions).
int orc_reaction_step(void* mech, const orc_options* o, int ncells, double* Y, double* T, double p,
                      double t0, const double* dt, double dt_scalar, double* Q, int* status,
                      long long* counters, int nthreads, const double* rho) {
  const orc::Mech& m = *(const orc::Mech*)mech;
  const int NC = m.nc;
  const unsigned NEQ = NC + 1;
  int nerr = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  const bool seq = o->sequential_state != 0;
#pragma omp parallel if (!seq) reduction(+ : nerr)
  {
    orc::Reactor reactor(m);
    orc::Gear g(reactor, NEQ);
    g.alfa2_[4] = o->alfa2_4; g.alfa2_[5] = o->alfa2_5; g.maximum_order_ = o->maximum_order;
    std::vector<double> y0(NEQ), yf(NEQ);
#pragma omp for schedule(dynamic, 1)
    for (int cell = 0; cell < ncells; ++cell) {
      if (!seq) { g.alfa2_[4] = o->alfa2_4; g.alfa2_[5] = o->alfa2_5; g.maximum_order_ = o->maximum_order; }
      double* Yc = Y + (size_t)cell * NC;
      int st = 0;
      if (T[cell] > o->tmin_chem) {
        for (int i = 0; i < NC; ++i) y0[i] = Yc[i];
        y0[NC] = T[cell];
        double sum = 0.;
        for (int i = 0; i < NC; ++i) { if (y0[i] < 0.) y0[i] = 0.; sum += y0[i]; }
        for (int i = 0; i < NC; ++i) y0[i] /= sum;
        reactor.P0 = p;
        reactor.rho0 = rho ? rho[cell] : 0.;   // chemistry_DI.H:168-203: SetReactor(V, P, rhoCells[celli])
        reactor.energy = o->energy != 0;
        if (!reactor.energy) reactor.QR = 0.;
        g.set_initial_conditions(t0, y0.data());
        g.full_piv_ = o->full_pivoting != 0;
        g.abs_tol_ = o->atol; g.rel_tol_ = o->rtol;
        for (unsigned i = 0; i < NEQ; ++i) { g.minv_[i] = 0.; g.maxv_[i] = 1.; }
        g.minv_[NC] = o->y_min_T; g.maxv_[NC] = o->y_max_T;
        g.max_number_steps_ = (unsigned)o->max_steps;
        const double dtc = dt ? dt[cell] : dt_scalar;
        st = g.solve(t0 + dtc);
        yf = g.y_;
        if (Q) Q[cell] = reactor.QR;
        if (counters) for (int k = 0; k < orc::NCOUNT; ++k) counters[(size_t)cell * orc::NCOUNT + k] = g.cnt_[k];
        if (st < 0) nerr++;
      } else {
        for (int i = 0; i < NC; ++i) yf[i] = Yc[i];
        yf[NC] = T[cell];
        st = 0;
        if (counters) for (int k = 0; k < orc::NCOUNT; ++k) counters[(size_t)cell * orc::NCOUNT + k] = 0;
      }
      double s = 0.;
      for (int i = 0; i < NC; ++i) s += yf[i];
      for (int i = 0; i < NC; ++i) yf[i] /= s;
      for (int i = 0; i < NC; ++i) Yc[i] = yf[i];
      if (o->energy) T[cell] = yf[NC];
      if (status) status[cell] = st;
    }
  }
  return nerr;
}

// Source terms of the compact Strang scheme, chemistry_DI.H:236-281: from the
// state before (Y0, T0: the cell's fields as the step found them) and after
// (Yf, Tf: the step's normalised result), cell-major:
//   rho = p MW / R / Tf, MW and cp of the mixture at (Yf, Tf)
//   (ThermodynamicsMap_CHEMKIN.hpp:429-434, 436-455, 506-511),
//   RR_i = rho (Yf_i - Y0_i) / dt, RT = rho cp (Tf - T0) / dt; zero where dt <= 1e-14.
int orc_compact_sources(void* mech, int ncells, const double* Y0, const double* T0, const double* Yf,
                        const double* Tf, double p, const double* dt, double dt_scalar, int energy, double* RR,
                        double* RT) {
  const orc::Mech& m = *(const orc::Mech*)mech;
  const int NC = m.nc;
  const auto& MW = m.F("mw");
  const auto& TM = m.F("t_mid");
  const auto& CH = m.F("cp_ht");
  const auto& CL = m.F("cp_lt");
  for (int c = 0; c < ncells; ++c) {
    const double deltat = dt ? dt[c] : dt_scalar;
    const double* yf = Yf + (size_t)c * NC;
    const double* y0 = Y0 + (size_t)c * NC;
    double* rr = RR + (size_t)c * NC;
    if (!(deltat > 1e-14)) {
      for (int i = 0; i < NC; ++i) rr[i] = 0.;
      if (energy && RT) RT[c] = 0.;
      continue;
    }
    const double T = Tf[c];
    double u = 0.;
    for (int i = 0; i < NC; ++i) u += yf[i] / MW[i];
    const double mwmix = 1. / u;
    double cpmix = 0.;
    const double T2 = T * T, T3 = T2 * T, T4 = T3 * T;
    for (int i = 0; i < NC; ++i) {
      const double x = mwmix * yf[i] / MW[i];
      const double* a = T > TM[i] ? &CH[5 * i] : &CL[5 * i];
      cpmix += (a[0] + T * a[1] + T2 * a[2] + T3 * a[3] + T4 * a[4]) * x;
    }
    cpmix *= orc::R_J_KMOL;
    cpmix /= mwmix;
    const double rhomix = p * mwmix / orc::R_J_KMOL / T;
    for (int i = 0; i < NC; ++i) rr[i] = rhomix * (yf[i] - y0[i]) / deltat;
    if (energy && RT) RT[c] = rhomix * cpmix * (T - T0[c]) / deltat;
  }
  return 0;
}

// Formation-rate output fields, chemistry_DI.H:293-326: R_i MW_i [kg/m3/s] of
// every species at the state y = [Y_1..Y_NC, T] (the reactor's R() after the
// solver's last right-hand-side call, which is made at the state it returns).
int orc_formation_rates(void* mech, double P, const double* y, double* out) {
  const orc::Mech& m = *(const orc::Mech*)mech;
  orc::Reactor r(m);
  r.P0 = P;
  std::vector<double> dy(m.nc + 1);
  r.equations(y, dy.data());
  const auto& MW = m.F("mw");
  for (int i = 0; i < m.nc; ++i) out[i] = r.R[i] * MW[i];
  return 0;
}

// Steady solvers' linearised sources, solvers/laminarSMOKE/steady/linearModel.H:92-170 (reactionSourceTerms,
// reactionJacobian) as jacobianEvaluation.H:60-92 stores them.  y = [Y_1..Y_NC, T] of one cell.
int orc_steady_sources(void* mech, double P, const double* y, double* s_implicit, double* s_explicit) {
  const orc::Mech& m = *(const orc::Mech*)mech;
  const int NC = m.nc, NE = NC + 1;
  const auto& MW = m.F("mw");
  orc::Reactor r(m);
  r.P0 = P;
  r.energy = true;
  std::vector<double> yc(NE), dy(NE), S0(NE), Sp(NE), yp(y, y + NE);
  auto sources = [&](const double* yy, double* S) {   // reactionSourceTerms: omega = max(y, 0)
    for (int i = 0; i < NC; ++i) yc[i] = std::max(yy[i], 0.);
    yc[NC] = yy[NC];
    r.equations(yc.data(), dy.data());
    for (int i = 0; i < NC; ++i) S[i] = r.R[i] * MW[i];
    S[NC] = r.QR;
  };
  sources(y, S0.data());
  const double ZERO_DER = std::sqrt(orc::TINY_FLOAT);
  const double ETA2 = std::sqrt(orc::MACH_EPS_DOUBLE);
  const double TOLR = 1.e-7, TOLA = 1.e-12;
  for (int k = 0; k < NE; ++k) {
    const double hf = 1.;
    const double error_weight = 1. / (TOLA + TOLR * std::fabs(y[k]));
    double hJ = ETA2 * std::fabs(std::max(y[k], 1. / error_weight));
    const double hJf = hf / error_weight;
    hJ = std::max(hJ, hJf);
    hJ = std::max(hJ, ZERO_DER);
    const double d = std::min(hJ, 1.e-3 + 1e-3 * std::fabs(y[k]));
    const double udy = 1. / d;
    yp[k] += d;
    sources(yp.data(), Sp.data());
    const double J = (Sp[k] - S0[k]) * udy;
    yp[k] = y[k];
    s_implicit[k] = J;
    s_explicit[k] = S0[k] - J * y[k];
  }
  return 0;
}

// The steady solvers' default linearisation (sparseJacobian true): linearModel::reactionJacobianSparse
// (steady/linearModel.H:172-232).  Species entries of the diagonal: JacobianSparsityPatternMap::Jacobian
// (maps/JacobianSparsityPatternMap.hpp:427-560) at omega* = max(max(y, 0), 1e-13) times MW, i.e.
//   J_k = sum over reactions of (nu_prod - nu_reac)_k * [ lambda_f r_f / omega*_k - lambda_b r_b / omega*_k
//         + third body (r_f - r_b) c*_k / omega*_k (eff - 1) / M + fall-off (r_f - r_b) dG / G
//         + CABR (r_f - r_b) ]
// with each bracket term present where the reaction's orders, efficiencies or bath species name k, and the
// fall-off derivative a 1e-4 forward difference of FallOffReactionsCorrection in omega_k.  The T entry is the
// forward difference of the dense path.  species / energy: the speciesEquations / energyEquation switches.
int orc_steady_sources_sparse(void* mech, double P, const double* y, double* s_implicit, double* s_explicit,
                              int species, int energy) {
  const orc::Mech& m = *(const orc::Mech*)mech;
  const int NC = m.nc, NE = NC + 1, NR = m.nr;
  const auto& MW = m.F("mw");
  orc::Reactor r(m);
  r.P0 = P;
  r.energy = true;
  std::vector<double> yc(NE), dy(NE), S0(NE), Sp(NE), yp(y, y + NE), J(NE, 0.);
  auto sources = [&](const double* yy, double* S) {   // reactionSourceTerms: omega = max(y, 0)
    for (int i = 0; i < NC; ++i) yc[i] = std::max(yy[i], 0.);
    yc[NC] = yy[NC];
    r.equations(yc.data(), dy.data());
    for (int i = 0; i < NC; ++i) S[i] = r.R[i] * MW[i];
    S[NC] = r.QR;
  };
  sources(y, S0.data());
  if (species) {
    const double eps = 1.e-13;   // SetEpsilon(1e-13)
    const double T = y[NC];
    std::vector<double> om(NC), cs(NC), rf(NR), rb(NR), Jd(NC, 0.), net(NR);
    for (int i = 0; i < NC; ++i) {
      const double o = std::max(y[i], 0.);
      om[i] = (o > eps) ? o : eps;
    }
    double u = 0.;
    for (int i = 0; i < NC; ++i) u += om[i] / MW[i];
    const double MWs = 1. / u;
    const double cTs = P / orc::R_J_KMOL / T;
    const double rhos = cTs * MWs;
    for (int i = 0; i < NC; ++i) cs[i] = om[i] * rhos / MW[i];
    for (int i = 0; i < NC; ++i) r.c[i] = cs[i];
    r.P_ = P;
    r.h_over_RT(T);
    r.kin_set_T(T);
    r.reaction_rates(cTs);
    const auto& isrev = m.I("is_reversible");
    for (int j = 0; j < NR; ++j) rf[j] = r.kMod[j] * r.fwd[j];
    for (int j = 0; j < NR; ++j) rb[j] = isrev[j] ? r.rev[j] * r.kMod[j] : 0.;
    const auto& op = m.I("ford_ptr"); const auto& os = m.I("ford_species"); const auto& ov = m.F("ford_val");
    const auto& rp = m.I("reac_ptr"); const auto& rs = m.I("reac_species"); const auto& rn = m.F("reac_nu");
    const auto& pp = m.I("prod_ptr"); const auto& ps = m.I("prod_species"); const auto& pn = m.F("prod_nu");
    const auto& tbr = m.I("tb_rxn"); const auto& tbp = m.I("tb_ptr");
    const auto& tbs = m.I("tb_species"); const auto& tbe = m.F("tb_eff_m1");
    const auto& fr = m.I("fo_rxn"); const auto& fsg = m.I("fo_single");
    const auto& fp = m.I("fo_ptr"); const auto& fs = m.I("fo_species");
    std::vector<double> cplus(cs);
    for (int k = 0; k < NC; ++k) {
      std::fill(net.begin(), net.end(), 0.);
      for (int j = 0; j < NR; ++j)
        for (int q = op[j]; q < op[j + 1]; ++q)
          if (os[q] == k) net[j] = ov[q] * rf[j] / om[k];
      for (int j = 0; j < NR; ++j)
        for (int q = pp[j]; q < pp[j + 1]; ++q)
          if (ps[q] == k) net[j] -= pn[q] * rb[j] / om[k];
      for (size_t sidx = 0; sidx < tbr.size(); ++sidx)
        for (int q = tbp[sidx]; q < tbp[sidx + 1]; ++q)
          if (tbs[q] == k) {
            const int j = tbr[sidx];
            net[j] += (rf[j] - rb[j]) * cs[k] / om[k] * tbe[q] / r.Mtb[sidx];
          }
      for (size_t f = 0; f < fr.size(); ++f) {
        bool has = fsg[f] == k;
        if (fsg[f] < 0)
          for (int q = fp[f]; q < fp[f + 1]; ++q) if (fs[q] == k) has = true;
        if (!has) continue;
        const int j = fr[f];
        const bool cabr = m.i.count("fo_cabr") && m.I("fo_cabr")[f] != 0;
        if (cabr) {
          net[j] += (rf[j] - rb[j]);
        } else {
          const double fo_eps = 1.e-4;
          cplus[k] = (om[k] + fo_eps) * rhos / MW[k];
          const double G = r.falloff_correction((int)f, cTs, cs.data());
          const double Gp = r.falloff_correction((int)f, cTs, cplus.data());
          const double dG = (Gp - G) / fo_eps;
          cplus[k] = om[k] * rhos / MW[k];
          net[j] += (rf[j] - rb[j]) * dG / G;
        }
      }
      for (int j = 0; j < NR; ++j)
        for (int q = rp[j]; q < rp[j + 1]; ++q)
          if (rs[q] == k) Jd[k] -= rn[q] * net[j];
      for (int j = 0; j < NR; ++j)
        for (int q = pp[j]; q < pp[j + 1]; ++q)
          if (ps[q] == k) Jd[k] += pn[q] * net[j];
    }
    for (int i = 0; i < NC; ++i) J[i] = Jd[i] * MW[i];
  }
  if (energy) {   // the dense path's forward difference, for T only (linearModel.H:195-230)
    const double ZERO_DER = std::sqrt(orc::TINY_FLOAT);
    const double ETA2 = std::sqrt(orc::MACH_EPS_DOUBLE);
    const double TOLR = 1.e-7, TOLA = 1.e-12;
    const int kd = NC;
    sources(y, S0.data());
    const double hf = 1.;
    const double error_weight = 1. / (TOLA + TOLR * std::fabs(y[kd]));
    double hJ = ETA2 * std::fabs(std::max(y[kd], 1. / error_weight));
    const double hJf = hf / error_weight;
    hJ = std::max(hJ, hJf);
    hJ = std::max(hJ, ZERO_DER);
    const double d = std::min(hJ, 1.e-3 + 1e-3 * std::fabs(y[kd]));
    const double udy = 1. / d;
    yp[kd] += d;
    sources(yp.data(), Sp.data());
    J[kd] = (Sp[kd] - S0[kd]) * udy;
    yp[kd] = y[kd];
  }
  for (int k = 0; k < NE; ++k) {
    s_implicit[k] = J[k];
    s_explicit[k] = S0[k] - J[k] * y[k];
  }
  return 0;
}

// DRG-reduced reaction step, solvers/laminarSMOKE/unsteady/chemistry_DRG.H:78-200, cells in order.
// Per cell above min_T: the analysis at the cell's concentrations (epsilon from the first band whose
// temperature is above the cell's; with none, the epsilon of the previous analysis stays), then the
// reduced system from t0 to t0 + dt with a new solver, the other species kept, the mass fractions
// normalised after the step.  The reference declares the solver inside the cell loop and applies the
// tolerances and bounds (T in [200, 6000]) only when celli == 0; every other cell integrates with the
// solver's defaults (absolute 1e-10, relative 100 * FLT_EPSILON, no bounds).  first_cell_options_only
// = 1 restates that; 0 gives every cell the options.  n_species / n_reactions: the drg fields (0 for
// skipped cells).
struct orc_drg_options {
  const int* key;
  int nkey;
  const double* band_T;
  const double* band_eps;
  int nbands;
  double epsilon0;
  double min_T;
  int first_cell_options_only;
};

int orc_reaction_step_drg(void* mech, const orc_options* o, const orc_drg_options* d, int ncells, double* Y,
                          double* T, double p, double t0, const double* dt, double dt_scalar, double* Q, int* status,
                          long long* counters, int* n_species, int* n_reactions) {
  const orc::Mech& m = *(const orc::Mech*)mech;
  const int NC = m.nc, NR = m.nr;
  const auto& MW = m.F("mw");
  orc::Reactor reactor(m);
  orc::Drg drg(m);
  std::vector<int> key(d->key, d->key + d->nkey), imp, drop;
  std::vector<double> omega(NC), x(NC), c(NC), yff(NC + 1);
  double eps = d->epsilon0;
  int nerr = 0;
  for (int cell = 0; cell < ncells; ++cell) {
    double* Yc = Y + (size_t)cell * NC;
    int st = 0;
    int nsp = 0, nrx = 0;
    if (T[cell] > d->min_T) {
      for (int i = 0; i < NC; ++i) omega[i] = Yc[i];
      double u = 0.;
      for (int i = 0; i < NC; ++i) u += omega[i] / MW[i];
      const double MWmix = 1. / u;
      for (int i = 0; i < NC; ++i) x[i] = MWmix * omega[i];
      for (int i = 0; i < NC; ++i) x[i] = x[i] / MW[i];
      const double cTot = p / orc::R_J_KMOL / T[cell];
      for (int i = 0; i < NC; ++i) c[i] = cTot * x[i];
      for (int b = 0; b < d->nbands; ++b)
        if (T[cell] < d->band_T[b]) { eps = d->band_eps[b]; break; }
      drg.analysis(reactor, T[cell], p, c.data(), eps, key, imp, drop);
      const int ni = (int)imp.size();
      const unsigned NEQ = ni + 1;
      std::vector<double> y0(NEQ);
      for (int i = 0; i < ni; ++i) y0[i] = omega[imp[i]];
      y0[ni] = T[cell];
      reactor.P0 = p;
      reactor.rho0 = 0.;
      reactor.energy = o->energy != 0;
      if (!reactor.energy) reactor.QR = 0.;
      reactor.omega = omega;
      reactor.drg_species = &imp;
      reactor.drg_dropped = &drop;
      orc::Gear g(reactor, NEQ);
      g.set_initial_conditions(t0, y0.data());
      if (cell == 0 || !d->first_cell_options_only) {
        g.full_piv_ = o->full_pivoting != 0;
        g.abs_tol_ = o->atol; g.rel_tol_ = o->rtol;
        for (unsigned i = 0; i < NEQ; ++i) { g.minv_[i] = 0.; g.maxv_[i] = 1.; }
        g.minv_[ni] = 200.; g.maxv_[ni] = 6000.;
      } else {
        g.abs_tol_ = 1.e-10; g.rel_tol_ = 100. * orc::MACH_EPS_FLOAT;   // MultiValueSolver.hpp:41-43
        g.min_c_ = false; g.max_c_ = false;
      }
      const double dtc = dt ? dt[cell] : dt_scalar;
      st = g.solve(t0 + dtc);
      reactor.drg_species = nullptr;
      reactor.drg_dropped = nullptr;
      for (int i = 0; i < NC; ++i) yff[i] = omega[i];
      yff[NC] = g.y_[ni];
      for (int i = 0; i < ni; ++i) yff[imp[i]] = g.y_[i];
      double sum = 0.;
      for (int i = 0; i < NC; ++i) sum += yff[i];
      for (int i = 0; i < NC; ++i) yff[i] /= sum;
      for (int i = 0; i < NC; ++i) Yc[i] = yff[i];
      if (o->energy) T[cell] = yff[NC];
      if (Q) Q[cell] = reactor.QR;
      if (counters) for (int k = 0; k < orc::NCOUNT; ++k) counters[(size_t)cell * orc::NCOUNT + k] = g.cnt_[k];
      nsp = ni;
      nrx = NR - (int)drop.size();
      if (st < 0) nerr++;
    } else if (counters) {
      for (int k = 0; k < orc::NCOUNT; ++k) counters[(size_t)cell * orc::NCOUNT + k] = 0;
    }
    if (status) status[cell] = st;
    if (n_species) n_species[cell] = nsp;
    if (n_reactions) n_reactions[cell] = nrx;
  }
  return nerr;
}

// The analysis alone at one state: important species (ascending) and dropped reactions.
int orc_drg_analysis(void* mech, double T, double P, const double* c, double eps, const int* key, int nkey,
                     int* important, int* n_important, int* dropped, int* n_dropped) {
  const orc::Mech& m = *(const orc::Mech*)mech;
  orc::Reactor reactor(m);
  orc::Drg drg(m);
  std::vector<int> k(key, key + nkey), imp, drop;
  drg.analysis(reactor, T, P, c, eps, k, imp, drop);
  for (size_t i = 0; i < imp.size(); ++i) important[i] = imp[i];
  for (size_t i = 0; i < drop.size(); ++i) dropped[i] = drop[i];
  *n_important = (int)imp.size();
  *n_dropped = (int)drop.size();
  return 0;
}

int orc_num_counters() { return orc::NCOUNT; }

}  // extern "C"
