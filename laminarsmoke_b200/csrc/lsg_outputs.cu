// Output fields of the reaction step beyond Y, T and Q, from laminarSMOKE's
// solvers/laminarSMOKE/unsteady/chemistry_DI.H:
//
// * the source terms of the compact Strang scheme (:236-281): the step leaves
//   the fields alone and hands the transport equations
//     RR_i = rho (Yf_i - Y0_i) / dt   and   RT = rho cp (Tf - T0) / dt,
//   rho and cp of the mixture at the step's result (Yf, Tf);
// * the formation-rate fields (:293-326): R_i MW_i [kg/m3/s] at a state.
//
// Thread per cell over species-major arrays: every species row is read with
// consecutive cells in consecutive lanes (coalesced), and each cell's sums run
// in species order.  HBM-bound: (3 NC + 3) doubles move per cell for the
// sources.  Compiled with FMA contraction off so each expression rounds like
// the reference's host arithmetic.
#include "lsg_common.cuh"
#include "lsg_kernels.h"

namespace lsg {

__global__ void __launch_bounds__(256) compact_sources_kernel(MechLayout L, const unsigned char* mech_gmem,
                                                              long ncells, const double* __restrict__ Y0,
                                                              const double* __restrict__ T0,
                                                              const double* __restrict__ Yf,
                                                              const double* __restrict__ Tf, long ld, double p,
                                                              const double* __restrict__ dt, double dt_scalar,
                                                              int energy, double* __restrict__ RR,
                                                              double* __restrict__ RT) {
  const MechView M{(const double*)mech_gmem, (const int*)(mech_gmem + (size_t)L.n_double * sizeof(double))};
  const double* MW = M.D(L.mw);
  const double* TM = M.D(L.t_mid);
  const int NC = L.nc;
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < ncells; c += (long)gridDim.x * blockDim.x) {
    const double deltat = dt ? dt[c] : dt_scalar;
    if (!(deltat > 1e-14)) {
      for (int i = 0; i < NC; ++i) RR[(long)i * ld + c] = 0.;
      if (energy && RT) RT[c] = 0.;
      continue;
    }
    const double T = Tf[c];
    // ThermodynamicsMap_CHEMKIN::MoleFractions_From_MassFractions (:429-434)
    double u = 0.;
    for (int i = 0; i < NC; ++i) u += Yf[(long)i * ld + c] / MW[i];
    const double mwmix = 1. / u;
    const double rhomix = p * mwmix / kRgas / T;
    for (int i = 0; i < NC; ++i) RR[(long)i * ld + c] = rhomix * (Yf[(long)i * ld + c] - Y0[(long)i * ld + c]) / deltat;
    if (energy && RT) {
      // cp_over_R (:436-455) and cpMolar_Mixture_From_MoleFractions (:506-511), per unit mass
      const double T2 = T * T, T3 = T2 * T, T4 = T3 * T;
      double cpmix = 0.;
      for (int i = 0; i < NC; ++i) {
        const double x = mwmix * Yf[(long)i * ld + c] / MW[i];
        const double* a = T > TM[i] ? M.D(L.cp_ht) + 5 * i : M.D(L.cp_lt) + 5 * i;
        cpmix += (a[0] + T * a[1] + T2 * a[2] + T3 * a[3] + T4 * a[4]) * x;
      }
      cpmix *= kRgas;
      cpmix /= mwmix;
      RT[c] = rhomix * cpmix * (T - T0[c]) / deltat;
    }
  }
}

// y = [Y; T] with leading dimension ncells, gathered from the caller's arrays.
__global__ void __launch_bounds__(256) gather_state_kernel(int nc, long ncells, const double* __restrict__ Y,
                                                           const double* __restrict__ T, long ld,
                                                           double* __restrict__ y) {
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < ncells; c += (long)gridDim.x * blockDim.x) {
    for (int i = 0; i < nc; ++i) y[(long)i * ncells + c] = Y[(long)i * ld + c];
    y[(long)nc * ncells + c] = T[c];
  }
}

// R_i MW_i = rho dY_i/dt, rho = cTot MW of the mixture computed as the
// right-hand side computes it (BatchReactorHomogeneousConstantPressure.H:175-223).
__global__ void __launch_bounds__(256) formation_rates_kernel(MechLayout L, const unsigned char* mech_gmem,
                                                              long ncells, const double* __restrict__ y,
                                                              const double* __restrict__ dy, double p,
                                                              double* __restrict__ out, long ld_out) {
  const MechView M{(const double*)mech_gmem, (const int*)(mech_gmem + (size_t)L.n_double * sizeof(double))};
  const double* MW = M.D(L.mw);
  const int NC = L.nc;
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < ncells; c += (long)gridDim.x * blockDim.x) {
    double u = 0.;
    for (int i = 0; i < NC; ++i) u += y[(long)i * ncells + c] / MW[i];
    const double MWmix = 1. / u;
    const double cTot = p / kRgas / y[(long)NC * ncells + c];
    const double rho = cTot * MWmix;
    for (int i = 0; i < NC; ++i) out[(long)i * ld_out + c] = rho * dy[(long)i * ncells + c];
  }
}

namespace {
unsigned grid_for(long ncells, int sm_count) {
  const long want = (ncells + 255) / 256;
  const long cap = (long)sm_count * 8;
  return (unsigned)(want < cap ? want : cap);
}
}  // namespace

cudaError_t launch_compact_sources(const MechLayout& L, const unsigned char* mech_gmem, long ncells,
                                   const double* Y0, const double* T0, const double* Yf, const double* Tf, long ld,
                                   double p, const double* dt, double dt_scalar, int energy, double* RR, double* RT,
                                   int sm_count, cudaStream_t stream) {
  if (ncells <= 0) return cudaSuccess;
  compact_sources_kernel<<<grid_for(ncells, sm_count), 256, 0, stream>>>(L, mech_gmem, ncells, Y0, T0, Yf, Tf, ld,
                                                                          p, dt, dt_scalar, energy, RR, RT);
  return cudaGetLastError();
}

cudaError_t launch_gather_state(int nc, long ncells, const double* Y, const double* T, long ld, double* y,
                                int sm_count, cudaStream_t stream) {
  if (ncells <= 0) return cudaSuccess;
  gather_state_kernel<<<grid_for(ncells, sm_count), 256, 0, stream>>>(nc, ncells, Y, T, ld, y);
  return cudaGetLastError();
}

cudaError_t launch_formation_rates(const MechLayout& L, const unsigned char* mech_gmem, long ncells,
                                   const double* y, const double* dy, double p, double* out, long ld_out,
                                   int sm_count, cudaStream_t stream) {
  if (ncells <= 0) return cudaSuccess;
  formation_rates_kernel<<<grid_for(ncells, sm_count), 256, 0, stream>>>(L, mech_gmem, ncells, y, dy, p, out,
                                                                          ld_out);
  return cudaGetLastError();
}

}  // namespace lsg
