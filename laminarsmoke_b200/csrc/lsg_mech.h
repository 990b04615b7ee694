// Device-side mechanism layout shared by the host runtime and the kernels.
//
// The packed blob (named arrays) is flattened on the host into ONE buffer:
// a double region followed by an int region.  Every array starts on a
// 16-byte boundary so the whole table (or any array of it) can be moved by a
// bulk copy.  Offsets are in elements of the region they live in.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define LSG_HD __host__ __device__
#else
#define LSG_HD
#endif

namespace lsg {

struct MechLayout {
  int nc, nr;                 // species, reactions
  int n_tb, n_fo, n_rev_th, n_rev_ex;
  int nnz_reac, nnz_prod, nnz_fr, nnz_tb, nnz_fo;
  int n_double, n_int;        // region sizes (elements, padded)
  uint32_t bytes;             // total bytes of the flattened buffer
  // ---- double region offsets
  int mw, cp_ht, cp_lt, dh_ht, dh_lt, ds_ht, ds_lt, t_mid;   // species
  int lnA, beta, eor, dnu;                                   // reactions
  int rev_lnA, rev_beta, rev_eor;                            // explicit reverse (by slot)
  int fo_lnA, fo_beta, fo_eor, fo_a, fo_b, fo_c, fo_d, fo_e; // fall-off (by slot)
  int reac_nu, prod_nu, fr_coef, tb_eff, fo_eff;             // CSR values
  int ford_val;                                              // forward rate-law orders (FORD or reac_nu)
  int plog_p, plog_lnp, plog_lnA, plog_beta, plog_eor;       // pressure-logarithmic points (by slot CSR)
  int n_plog;                                                // reactions with PLOG
  int cheb_coef, cheb_lim;                                   // Chebyshev coefficients, limits (by slot)
  int n_cheb;                                                // reactions with CHEB
  // extended PLOG (PLOGMX / PLOGSP): per slot a CSR of baths, per bath a CSR of points
  int xplog_p, xplog_lnp, xplog_lnA, xplog_beta, xplog_eor;  // points
  int n_xplog;                                               // reactions with extended PLOG
  // extended fall-off (LOWMX / LOWSP): k_inf (A, beta, E/R) per slot, per bath k0 (A, beta, E/R), form, params
  int xfo_kinf, xfo_tb_eff, xfo_low, xfo_par;
  int n_xfo;                                                 // reactions with extended fall-off
  // ---- int region offsets
  int a_sign, rev_kind, rev_slot, tb_slot, fo_slot;          // per reaction
  int reac_ptr, reac_sp, prod_ptr, prod_sp;                  // per reaction CSR
  int ford_ptr, ford_sp;                                     // per reaction CSR of the forward orders
  int plog_slot, plog_ptr, plog_rxn;                         // per reaction slot (-1: none); CSR by slot
  int cheb_slot, cheb_rxn, cheb_nm, cheb_ptr;                // likewise for Chebyshev reactions
  int xplog_slot, xplog_bath_ptr, xplog_bath_sp, xplog_ptr;  // per reaction slot (-1: none); baths (-1: mixture)
  int xfo_slot, xfo_tb_ptr, xfo_tb_sp, xfo_bath_ptr, xfo_bath_sp, xfo_type, xfo_par_ptr;
  int fr_ptr, fr_rxn;                                        // per species CSR
  int tb_ptr, tb_sp;                                         // third body CSR (by slot)
  int fo_type, fo_single, fo_ptr, fo_sp;                     // fall-off (by slot)
  int fo_cabr;                                               // 1: chemically activated bimolecular (by slot)
};

// Fitted transport properties (the packed blob's tr_* arrays), flattened into
// a table of their own: [double region][int region], offsets in elements.
// Only the property update reads it, so the kinetics table stays as small as
// the reaction kernels need.
struct TransportLayout {
  int nc, n_pair, n_teta;     // species, pairs j < k, light species with thermal-diffusion ratios
  int n_double, n_int;
  uint32_t bytes;
  // ---- double region
  int eta, lam;               // [nc][4]: ln(eta), ln(lambda) in powers of ln T
  int gam;                    // [n_pair][4]: ln(D_jk P) [m2/s bar] in powers of ln T, pairs j < k row by row
  int teta;                   // [n_teta][nc][4]: theta_ij in powers of T
  int wilke_phi;              // [nc][nc]: 1 / sqrt(8 (1 + M_k / M_j))
  int wilke_r14;              // [nc][nc]: (M_j / M_k)^(1/4)
  // ---- int region
  int iteta;                  // [n_teta] species index of each light species
};

// Views into a flattened table (global or shared memory).
struct MechView {
  const double* d;
  const int* i;
  LSG_HD const double* D(int off) const { return d + off; }
  LSG_HD const int* I(int off) const { return i + off; }
};

}  // namespace lsg
