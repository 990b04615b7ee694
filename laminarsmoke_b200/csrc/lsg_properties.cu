// Per-cell property update after the reaction step: laminarSMOKE's loop over
// the cells in solvers/laminarSMOKE/properties.H:40-190, with the mixture
// rules of OpenSMOKE++'s maps:
//
// * x_i = MWmix Y_i / MW_i, MWmix = 1 / sum Y_i / MW_i
//   (ThermodynamicsMap_CHEMKIN.hpp:429-434);
// * cTot = p / (R T), psi = cTot MWmix / p, h = R T sum x_i (h/RT)_i / MWmix
//   (properties.H:93-96, ThermodynamicsMap_CHEMKIN.hpp:514-520);
// * mu: Wilke's rule over the fitted species viscosities, pairs k < j in the
//   reference's order (TransportPropertiesMap_CHEMKIN.hpp:729-766, 959-1001);
// * lambda: Mathur-Saxena, 0.5 (sum x lambda + 1 / sum x / lambda) (:947-957);
//   cp = sum x cp_i / MWmix, cv = (cp_molar - R) / MWmix, species cp_i / MW_i
//   (properties.H:103-122), evaluated when the energy equation is solved or
//   the Lewis-number diffusivities need them;
// * the simplified transport option mu0 (T/T0)^beta0, mu cp / Pr0 (:124-133);
// * Dmix: mixture-averaged, (MW~ - x~_k M_k) / (MW~ sum_j x~_j / D_kj) with
//   x~ = (x + 1e-14) / (1 + 1e-14 nc) and D_kj from the binary fits at the
//   cell's pressure (gamma :798-859, gammaMix :1032-1059); or
//   lambda / (p psi cp Le_k) with Lewis numbers (properties.H:152-162);
// * Dsoret_i = Dmix_i theta_i MW_i / MWmix, theta_i = sum_j theta_ij x_i x_j
//   for the light species (teta :768-796, tetaMix :1103-1117;
//   properties.H:177-189).
//
// One thread per cell.  Species rows are species-major with the cells of a
// warp in consecutive lanes, so every row read and written is coalesced.  The
// per-species work arrays of a cell (x, sqrt eta, the Wilke / diffusion sums)
// sit in shared memory laid out [array][species][thread], so the lanes of a
// warp touch consecutive doubles; three arrays keep about 20 warps resident per
// SM at 14 species.  The pair loops are O(nc^2) per cell and read the
// mechanism's fit and Wilke tables as warp-uniform loads.  The kernel is bound
// by its FP64 arithmetic (exponentials and divisions of the pair loops), not
// by HBM.  Compiled with FMA contraction off so each expression rounds like the
// host arithmetic.
#include "lsg_common.cuh"
#include "lsg_kernels.h"

namespace lsg {

namespace {
constexpr int kPropArrays = 3;              // x, sqrt(eta), sums
constexpr size_t kPropSmemMax = 200 * 1024;
constexpr double kThreshold = 1.e-14;       // TransportPropertiesMap_CHEMKIN.hpp:47
constexpr double kMu0 = 1.8405e-5, kT0 = 300., kBeta0 = 0.6759, kPr0 = 0.7;   // properties.H:126-129

size_t prop_smem(int nc, int bd) { return (size_t)kPropArrays * nc * bd * sizeof(double); }
}  // namespace

int properties_block(int nc) {
  for (int bd : {128, 64, 32})
    if (prop_smem(nc, bd) <= (bd == 32 ? kPropSmemMax : 64 * 1024)) return bd;
  return 0;
}

__global__ void __launch_bounds__(128) properties_kernel(MechLayout L, const unsigned char* mech_gmem,
                                                         TransportLayout TL, const unsigned char* tr_gmem,
                                                         PropArgs a) {
  extern __shared__ double sm[];
  const int nc = L.nc;
  const int bd = blockDim.x;
  const long c = blockIdx.x * (long)bd + threadIdx.x;
  if (c >= a.ncells) return;   // no block barriers below
  const MechView M{(const double*)mech_gmem, (const int*)(mech_gmem + (size_t)L.n_double * sizeof(double))};
  const double* TD = (const double*)tr_gmem;
  const int* TI = (const int*)(tr_gmem + (size_t)TL.n_double * sizeof(double));
  const double* MW = M.D(L.mw);
  const double* TM = M.D(L.t_mid);
  double* xs = sm + threadIdx.x;             // xs[s * bd]
  double* ss = xs + (size_t)nc * bd;
  double* acc = ss + (size_t)nc * bd;
  const long ld = a.ld, lo = a.ld_out;

  const double T = a.T[c];
  const double p = a.p ? a.p[c] : a.p_scalar;
  double u = 0.;
  for (int s = 0; s < nc; ++s) u += a.Y[s * ld + c] / MW[s];
  const double MWm = 1. / u;
  for (int s = 0; s < nc; ++s) {
    const double x = MWm * a.Y[s * ld + c] / MW[s];
    xs[(size_t)s * bd] = x;
    if (a.X) a.X[s * lo + c] = x;
  }
  const double cTot = p / kRgas / T;
  const double psi = cTot * MWm / p;
  if (a.MWmix) a.MWmix[c] = MWm;
  if (a.cTot) a.cTot[c] = cTot;
  if (a.psi) a.psi[c] = psi;

  const double T2 = T * T, T3 = T2 * T, T4 = T3 * T, uT = 1. / T;
  if (a.h) {
    double hmix = 0.;
    for (int s = 0; s < nc; ++s) {
      const double* d = T > TM[s] ? M.D(L.dh_ht) + 6 * s : M.D(L.dh_lt) + 6 * s;
      const double hrt = d[0] + T * d[1] + T2 * d[2] + T3 * d[3] + T4 * d[4] + uT * d[5];
      hmix += hrt * xs[(size_t)s * bd];
    }
    hmix *= kRgas * T;
    a.h[c] = hmix / MWm;
  }

  const double lT = log(T), lT2 = lT * lT, lT3 = lT * lT2;
  // Wilke's rule (etaMix)
  const double* fe = TD + TL.eta;
  auto eta_of = [&](int s) {
    double sum = fe[4 * s];
    sum += fe[4 * s + 1] * lT;
    sum += fe[4 * s + 2] * lT2;
    sum += fe[4 * s + 3] * lT3;
    return exp(sum);
  };
  for (int s = 0; s < nc; ++s) {
    ss[(size_t)s * bd] = sqrt(eta_of(s));
    acc[(size_t)s * bd] = xs[(size_t)s * bd];
  }
  // Pair (k, j), k < j, adds x_j phi_kj (1 + d)^2 to sum_k and x_k phi_jk (1 + 1/d)^2 to
  // sum_j, d = sqrt(eta_k) / sqrt(eta_j) (M_j / M_k)^(1/4).  With j outermost each sum
  // receives its terms in the reference's order (the k < j terms, then j < k ascending),
  // and 1 / sqrt(eta_j) is formed once per species as there.
  const double* phi = TD + TL.wilke_phi;
  const double* r14 = TD + TL.wilke_r14;
  for (int j = 1; j < nc; ++j) {
    const double usj = 1. / ss[(size_t)j * bd], xj = xs[(size_t)j * bd];
    double sj = acc[(size_t)j * bd];
    for (int k = 0; k < j; ++k) {
      const double d = ss[(size_t)k * bd] * usj * r14[k * nc + j];
      acc[(size_t)k * bd] += xj * phi[k * nc + j] * (1. + d) * (1. + d);
      sj += xs[(size_t)k * bd] * phi[j * nc + k] * (1. + 1. / d) * (1. + 1. / d);
    }
    acc[(size_t)j * bd] = sj;
  }
  double mu = 0.;
  for (int s = 0; s < nc; ++s) mu += xs[(size_t)s * bd] * eta_of(s) / acc[(size_t)s * bd];

  const bool lewis = a.lewis != nullptr;
  double lambda = 0., cp = 0.;
  if (a.energy || lewis) {
    const double* fl = TD + TL.lam;
    double s1 = 0., s2 = 0.;
    for (int s = 0; s < nc; ++s) {
      double sum = fl[4 * s];
      sum += fl[4 * s + 1] * lT;
      sum += fl[4 * s + 2] * lT2;
      sum += fl[4 * s + 3] * lT3;
      const double l = exp(sum);
      s1 += xs[(size_t)s * bd] * l;
      s2 += xs[(size_t)s * bd] / l;
    }
    lambda = 0.50 * (s1 + 1. / s2);
    double cpm = 0.;
    for (int s = 0; s < nc; ++s) {
      const double* q = T > TM[s] ? M.D(L.cp_ht) + 5 * s : M.D(L.cp_lt) + 5 * s;
      const double cpr = q[0] + T * q[1] + T2 * q[2] + T3 * q[3] + T4 * q[4];
      cpm += cpr * xs[(size_t)s * bd];
      if (a.cp_species) a.cp_species[s * lo + c] = (cpr * kRgas) / MW[s];
    }
    cpm *= kRgas;
    if (a.cv) a.cv[c] = (cpm - kRgas) / MWm;
    cp = cpm / MWm;
    if (a.cp) a.cp[c] = cp;
  }
  if (a.simplified) {
    mu = kMu0 * pow(T / kT0, kBeta0);
    lambda = mu * cp / kPr0;
  }
  if (a.mu) a.mu[c] = mu;
  if ((a.energy || lewis) && a.lambda) a.lambda[c] = lambda;

  if (!a.Dmix) return;
  if (lewis) {
    const double coef = lambda / (p * psi) / cp;
    for (int s = 0; s < nc; ++s) {
      const double D = coef / a.lewis[s];
      acc[(size_t)s * bd] = D;
      a.Dmix[s * lo + c] = D;
    }
  } else {
    const double pbar = p / 100000.;
    const double sum_thr = 1. + kThreshold * (double)nc;
    double MWc = 0.;
    for (int s = 0; s < nc; ++s) {
      MWc += ((xs[(size_t)s * bd] + kThreshold) / sum_thr) * MW[s];
      acc[(size_t)s * bd] = 0.;
    }
    const double* fg = TD + TL.gam;
    int q = 0;
    for (int k = 0; k < nc; ++k) {
      const double xk = (xs[(size_t)k * bd] + kThreshold) / sum_thr;
      double sk = acc[(size_t)k * bd];
      for (int j = k + 1; j < nc; ++j, ++q) {
        double sum = fg[4 * q];
        sum += fg[4 * q + 1] * lT;
        sum += fg[4 * q + 2] * lT2;
        sum += fg[4 * q + 3] * lT3;
        const double g = pbar / exp(sum);
        acc[(size_t)j * bd] += xk * g;
        sk += ((xs[(size_t)j * bd] + kThreshold) / sum_thr) * g;
      }
      acc[(size_t)k * bd] = sk;
    }
    for (int s = 0; s < nc; ++s) {
      const double xc = (xs[(size_t)s * bd] + kThreshold) / sum_thr;
      const double D = (MWc - xc * MW[s]) / (MWc * acc[(size_t)s * bd]);
      acc[(size_t)s * bd] = D;
      a.Dmix[s * lo + c] = D;
    }
  }
  if (!a.Dsoret) return;
  const double* ft = TD + TL.teta;
  const int* it = TI + TL.iteta;
  for (int m = 0; m < TL.n_teta; ++m) {
    const int i = it[m];
    const double xi = xs[(size_t)i * bd];
    double th = 0.;
    for (int j = 0; j < nc; ++j) {
      const double* f = ft + 4 * ((size_t)m * nc + j);
      double sum = f[0];
      sum += f[1] * T;
      sum += f[2] * T2;
      sum += f[3] * T3;
      th += sum * xi * xs[(size_t)j * bd];
    }
    a.Dsoret[m * lo + c] = acc[(size_t)i * bd] * th * MW[i] / MWm;
  }
}

cudaError_t launch_properties(const MechLayout& L, const unsigned char* mech_gmem, const TransportLayout& TL,
                              const unsigned char* tr_gmem, const PropArgs& a, cudaStream_t stream) {
  if (a.ncells <= 0) return cudaSuccess;
  const int bd = properties_block(L.nc);
  if (bd == 0) return cudaErrorInvalidValue;
  const size_t smem = prop_smem(L.nc, bd);
  const cudaError_t e =
      cudaFuncSetAttribute(properties_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPropSmemMax);
  if (e != cudaSuccess) return e;
  const long grid = (a.ncells + bd - 1) / bd;
  properties_kernel<<<(unsigned)grid, bd, smem, stream>>>(L, mech_gmem, TL, tr_gmem, a);
  return cudaGetLastError();
}

}  // namespace lsg
