// Host side: packed blob (named arrays) -> flattened device table (lsg_mech.h).
#include "lsg_mech_host.h"

#include <cmath>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace lsg {

namespace {
struct Blob {
  std::map<std::string, std::vector<double>> f;
  std::map<std::string, std::vector<int>> i;
  const std::vector<double>& F(const char* k) const {
    auto it = f.find(k);
    if (it == f.end()) throw std::runtime_error(std::string("mechanism blob: missing array ") + k);
    return it->second;
  }
  const std::vector<int>& I(const char* k) const {
    auto it = i.find(k);
    if (it == i.end()) throw std::runtime_error(std::string("mechanism blob: missing array ") + k);
    return it->second;
  }
};

bool parse(const unsigned char* p, size_t n, Blob& b, std::string& err) {
  if (n < 16 || std::memcmp(p, "LSMECH01", 8) != 0) { err = "bad magic"; return false; }
  uint32_t na;
  std::memcpy(&na, p + 8, 4);
  size_t pos = 16;
  for (uint32_t a = 0; a < na; ++a) {
    if (pos + 48 > n) { err = "truncated header"; return false; }
    char name[33];
    std::memcpy(name, p + pos, 32);
    name[32] = 0;
    uint32_t code;
    uint64_t count;
    std::memcpy(&code, p + pos + 32, 4);
    std::memcpy(&count, p + pos + 40, 8);
    pos += 48;
    if (code > 1) { err = "bad dtype"; return false; }
    const size_t item = code == 0 ? 8 : 4;
    if (count > (n - pos) / item) { err = "truncated payload"; return false; }   // no overflow of item * count
    const size_t nb = item * count;
    if (code == 0) {
      std::vector<double> v(count);
      if (nb) std::memcpy(v.data(), p + pos, nb);
      b.f[name] = std::move(v);
    } else {
      std::vector<int> v(count);
      if (nb) std::memcpy(v.data(), p + pos, nb);
      b.i[name] = std::move(v);
    }
    pos += nb + ((8 - nb % 8) % 8);
  }
  return true;
}

struct Builder {
  std::vector<double> d;
  std::vector<int> iv;
  int addd(const std::vector<double>& v) {
    while (d.size() % 2) d.push_back(0.);  // 16-byte alignment
    const int off = (int)d.size();
    d.insert(d.end(), v.begin(), v.end());
    return off;
  }
  int addi(const std::vector<int>& v) {
    while (iv.size() % 4) iv.push_back(0);
    const int off = (int)iv.size();
    iv.insert(iv.end(), v.begin(), v.end());
    return off;
  }
};
}  // namespace

// The transport fits, when the blob has them, with the Wilke factors of every
// species pair (TransportPropertiesMap_CHEMKIN.hpp:653-688) precomputed.
static bool build_transport(const Blob& b, int nc, HostMech& out, std::string& err) {
  out.has_transport = false;
  out.tbuffer.clear();
  out.iteta.clear();
  if (!b.f.count("tr_eta")) return true;
  const auto& eta = b.F("tr_eta");
  const auto& lam = b.F("tr_lambda");
  const auto& gam = b.F("tr_gamma");
  const auto& teta = b.F("tr_teta");
  const auto& it = b.I("tr_iteta");
  const long npair = (long)nc * (nc - 1) / 2;
  const long nt = (long)it.size();
  if ((long)eta.size() != 4L * nc || (long)lam.size() != 4L * nc || (long)gam.size() != 4 * npair ||
      (long)teta.size() != 4 * nt * nc) {
    err = "inconsistent transport arrays in mechanism blob";
    return false;
  }
  for (int v : it)
    if (v < 0 || v >= nc) { err = "transport species index out of range in mechanism blob"; return false; }
  const std::vector<double>& M = out.mw;
  std::vector<double> phi((size_t)nc * nc, 0.), r14((size_t)nc * nc, 0.);
  for (int k = 0; k < nc; ++k)
    for (int j = 0; j < nc; ++j) {
      phi[(size_t)k * nc + j] = 1. / std::sqrt(8. * (1. + M[k] / M[j]));
      r14[(size_t)k * nc + j] = std::sqrt(std::sqrt(M[j] / M[k]));
    }
  TransportLayout T{};
  T.nc = nc;
  T.n_pair = (int)npair;
  T.n_teta = (int)nt;
  Builder B;
  T.eta = B.addd(eta);
  T.lam = B.addd(lam);
  T.gam = B.addd(gam.empty() ? std::vector<double>(2, 0.) : gam);
  T.teta = B.addd(teta.empty() ? std::vector<double>(2, 0.) : teta);
  T.wilke_phi = B.addd(phi);
  T.wilke_r14 = B.addd(r14);
  T.iteta = B.addi(it.empty() ? std::vector<int>(1, 0) : it);
  while (B.d.size() % 2) B.d.push_back(0.);
  while (B.iv.size() % 4) B.iv.push_back(0);
  T.n_double = (int)B.d.size();
  T.n_int = (int)B.iv.size();
  T.bytes = (uint32_t)(B.d.size() * sizeof(double) + B.iv.size() * sizeof(int));
  out.tbuffer.resize(T.bytes);
  std::memcpy(out.tbuffer.data(), B.d.data(), B.d.size() * sizeof(double));
  std::memcpy(out.tbuffer.data() + B.d.size() * sizeof(double), B.iv.data(), B.iv.size() * sizeof(int));
  out.tlayout = T;
  out.iteta = it;
  out.has_transport = true;
  return true;
}

bool build_mechanism(const void* blob, size_t nbytes, HostMech& out, std::string& err) {
  Blob b;
  try {
    if (!parse((const unsigned char*)blob, nbytes, b, err)) return false;
  } catch (const std::exception& e) {
    err = std::string("mechanism blob: ") + e.what();
    return false;
  }
  try {
    const auto& dims = b.I("dims");
    const int nc = dims.at(0), nr = dims.at(1);
    if (nc <= 0 || nr < 0 || (int)b.F("mw").size() != nc || (int)b.F("lnA").size() != nr) {
      err = "bad dimensions";   // before anything is sized from nc or nr
      return false;
    }
    MechLayout L{};
    L.nc = nc;
    L.nr = nr;
    Builder B;
    L.mw = B.addd(b.F("mw"));
    L.cp_ht = B.addd(b.F("cp_ht"));
    L.cp_lt = B.addd(b.F("cp_lt"));
    L.dh_ht = B.addd(b.F("dh_ht"));
    L.dh_lt = B.addd(b.F("dh_lt"));
    L.ds_ht = B.addd(b.F("ds_ht"));
    L.ds_lt = B.addd(b.F("ds_lt"));
    L.t_mid = B.addd(b.F("t_mid"));
    L.lnA = B.addd(b.F("lnA"));
    L.beta = B.addd(b.F("beta"));
    L.eor = B.addd(b.F("e_over_r"));
    L.dnu = B.addd(b.F("delta_nu"));
    L.rev_lnA = B.addd(b.F("lnA_rev"));
    L.rev_beta = B.addd(b.F("beta_rev"));
    L.rev_eor = B.addd(b.F("e_over_r_rev"));
    L.fo_lnA = B.addd(b.F("fo_lnA"));
    L.fo_beta = B.addd(b.F("fo_beta"));
    L.fo_eor = B.addd(b.F("fo_e_over_r"));
    L.fo_a = B.addd(b.F("fo_a"));
    L.fo_b = B.addd(b.F("fo_b"));
    L.fo_c = B.addd(b.F("fo_c"));
    L.fo_d = B.addd(b.F("fo_d"));
    L.fo_e = B.addd(b.F("fo_e"));
    L.reac_nu = B.addd(b.F("reac_nu"));
    // forward rate-law orders: the FORD lists when the mechanism has them, else the reactant coefficients
    const bool ford = b.f.count("ford_val") != 0;
    const std::vector<int>& ford_ptr = ford ? b.I("ford_ptr") : b.I("reac_ptr");
    const std::vector<int>& ford_sp = ford ? b.I("ford_species") : b.I("reac_species");
    L.ford_val = B.addd(ford ? b.F("ford_val") : b.F("reac_nu"));
    L.prod_nu = B.addd(b.F("prod_nu"));
    L.fr_coef = B.addd(b.F("fr_coef"));
    L.tb_eff = B.addd(b.F("tb_eff_m1"));
    // pressure-logarithmic (PLOG) reactions, when the mechanism has them
    const bool plog = b.f.count("plog_p") != 0;
    const std::vector<double> none_d(2, 0.);
    const std::vector<int> none_i(2, 0), plog_ptr0{0};
    L.plog_p = B.addd(plog ? b.F("plog_p") : none_d);
    L.plog_lnp = B.addd(plog ? b.F("plog_lnp") : none_d);
    L.plog_lnA = B.addd(plog ? b.F("plog_lnA") : none_d);
    L.plog_beta = B.addd(plog ? b.F("plog_beta") : none_d);
    L.plog_eor = B.addd(plog ? b.F("plog_eor") : none_d);
    // Chebyshev reactions, when the mechanism has them
    const bool cheb = b.f.count("cheb_coef") != 0;
    L.cheb_coef = B.addd(cheb ? b.F("cheb_coef") : none_d);
    L.cheb_lim = B.addd(cheb ? b.F("cheb_lim") : none_d);
    L.fo_eff = B.addd(b.F("fo_eff_m1"));
    // extended PLOG and extended fall-off, when the mechanism has them
    const bool xplog = b.i.count("xplog_rxn") != 0;
    const bool xfo = b.i.count("xfo_rxn") != 0;
    L.xplog_p = B.addd(xplog ? b.F("xplog_p") : none_d);
    L.xplog_lnp = B.addd(xplog ? b.F("xplog_lnp") : none_d);
    L.xplog_lnA = B.addd(xplog ? b.F("xplog_lnA") : none_d);
    L.xplog_beta = B.addd(xplog ? b.F("xplog_beta") : none_d);
    L.xplog_eor = B.addd(xplog ? b.F("xplog_eor") : none_d);
    L.xfo_kinf = B.addd(xfo ? b.F("xfo_kinf") : none_d);
    L.xfo_tb_eff = B.addd(xfo && !b.F("xfo_tb_eff_m1").empty() ? b.F("xfo_tb_eff_m1") : none_d);
    L.xfo_low = B.addd(xfo ? b.F("xfo_low") : none_d);
    L.xfo_par = B.addd(xfo && !b.F("xfo_par").empty() ? b.F("xfo_par") : none_d);

    const auto& isrev = b.I("is_reversible");
    const auto& rth = b.I("rev_thermo");
    const auto& rex = b.I("rev_explicit");
    std::vector<int> rev_kind(nr, 0), rev_slot(nr, -1), tb_slot(nr, -1), fo_slot(nr, -1);
    for (size_t k = 0; k < rth.size(); ++k) { rev_kind.at(rth[k]) = 1; rev_slot.at(rth[k]) = (int)k; }
    for (size_t k = 0; k < rex.size(); ++k) { rev_kind.at(rex[k]) = 2; rev_slot.at(rex[k]) = (int)k; }
    for (int j = 0; j < nr; ++j)
      if (isrev.at(j) && rev_kind[j] == 0) { err = "reversible reaction without reverse data"; return false; }
    const auto& tbr = b.I("tb_rxn");
    const auto& fr = b.I("fo_rxn");
    for (size_t k = 0; k < tbr.size(); ++k) tb_slot.at(tbr[k]) = (int)k;
    for (size_t k = 0; k < fr.size(); ++k) fo_slot.at(fr[k]) = (int)k;

    std::vector<int> plog_slot(nr, -1);
    const std::vector<int> plog_rxn = plog ? b.I("plog_rxn") : std::vector<int>();
    const std::vector<int> plog_ptr = plog ? b.I("plog_ptr") : plog_ptr0;
    for (size_t k = 0; k < plog_rxn.size(); ++k) plog_slot.at(plog_rxn[k]) = (int)k;
    if (plog_ptr.size() != plog_rxn.size() + 1 || (plog && (size_t)plog_ptr.back() != b.F("plog_p").size())) {
      err = "inconsistent PLOG arrays in mechanism blob";
      return false;
    }
    for (size_t k = 0; k + 1 < plog_ptr.size(); ++k)
      if (plog_ptr[k + 1] <= plog_ptr[k]) { err = "PLOG reaction without points"; return false; }
    L.n_plog = (int)plog_rxn.size();
    L.plog_slot = B.addi(plog_slot);
    L.plog_ptr = B.addi(plog_ptr);
    L.plog_rxn = B.addi(plog_rxn.empty() ? none_i : plog_rxn);
    std::vector<int> cheb_slot(nr, -1);
    const std::vector<int> cheb_rxn = cheb ? b.I("cheb_rxn") : std::vector<int>();
    const std::vector<int> cheb_ptr = cheb ? b.I("cheb_ptr") : plog_ptr0;
    const std::vector<int> cheb_nm = cheb ? b.I("cheb_nm") : none_i;
    for (size_t k = 0; k < cheb_rxn.size(); ++k) cheb_slot.at(cheb_rxn[k]) = (int)k;
    if (cheb_ptr.size() != cheb_rxn.size() + 1 || (cheb && (cheb_nm.size() != 2 * cheb_rxn.size() ||
        (size_t)cheb_ptr.back() != b.F("cheb_coef").size() || b.F("cheb_lim").size() != 5 * cheb_rxn.size()))) {
      err = "inconsistent Chebyshev arrays in mechanism blob";
      return false;
    }
    for (size_t k = 0; k < cheb_rxn.size(); ++k)
      if (cheb_nm[2 * k] < 1 || cheb_nm[2 * k + 1] < 1 || cheb_ptr[k + 1] - cheb_ptr[k] != cheb_nm[2 * k] * cheb_nm[2 * k + 1]) {
        err = "inconsistent Chebyshev table in mechanism blob";
        return false;
      }
    L.n_cheb = (int)cheb_rxn.size();
    {
      // extended PLOG: slots, bath CSR (species or -1 for the mixture), point CSR per bath
      std::vector<int> xs(nr, -1);
      const std::vector<int> xr = xplog ? b.I("xplog_rxn") : std::vector<int>();
      const std::vector<int> bp = xplog ? b.I("xplog_bath_ptr") : plog_ptr0;
      const std::vector<int> bs = xplog ? b.I("xplog_bath_sp") : std::vector<int>();
      const std::vector<int> qp = xplog ? b.I("xplog_ptr") : plog_ptr0;
      for (size_t k = 0; k < xr.size(); ++k) {
        if (xr[k] < 0 || xr[k] >= nr || xs[xr[k]] >= 0) { err = "inconsistent extended PLOG arrays in mechanism blob"; return false; }
        xs[xr[k]] = (int)k;
      }
      bool okx = bp.size() == xr.size() + 1 && qp.size() == bs.size() + 1 && bp[0] == 0 && qp[0] == 0 &&
                 (size_t)bp.back() == bs.size() && (!xplog || (size_t)qp.back() == b.F("xplog_p").size());
      for (size_t k = 0; okx && k + 1 < bp.size(); ++k) okx = bp[k + 1] > bp[k];
      for (size_t k = 0; okx && k + 1 < qp.size(); ++k) okx = qp[k + 1] > qp[k];
      for (size_t k = 0; okx && k < bs.size(); ++k) okx = bs[k] >= -1 && bs[k] < nc;
      if (okx && xplog)
        for (const char* k : {"xplog_lnp", "xplog_lnA", "xplog_beta", "xplog_eor"})
          okx = okx && b.F(k).size() == b.F("xplog_p").size();
      if (!okx) { err = "inconsistent extended PLOG arrays in mechanism blob"; return false; }
      L.n_xplog = (int)xr.size();
      L.xplog_slot = B.addi(xs);
      L.xplog_bath_ptr = B.addi(bp);
      L.xplog_bath_sp = B.addi(bs.empty() ? none_i : bs);
      L.xplog_ptr = B.addi(qp);
    }
    {
      // extended fall-off: slots, third-body CSR, bath CSR, per bath form and parameter CSR
      std::vector<int> xs(nr, -1);
      const std::vector<int> xr = xfo ? b.I("xfo_rxn") : std::vector<int>();
      const std::vector<int> tp = xfo ? b.I("xfo_tb_ptr") : plog_ptr0;
      const std::vector<int> ts = xfo ? b.I("xfo_tb_sp") : std::vector<int>();
      const std::vector<int> bp = xfo ? b.I("xfo_bath_ptr") : plog_ptr0;
      const std::vector<int> bs = xfo ? b.I("xfo_bath_sp") : std::vector<int>();
      const std::vector<int> ty = xfo ? b.I("xfo_type") : std::vector<int>();
      const std::vector<int> pp = xfo ? b.I("xfo_par_ptr") : plog_ptr0;
      for (size_t k = 0; k < xr.size(); ++k) {
        if (xr[k] < 0 || xr[k] >= nr || xs[xr[k]] >= 0) { err = "inconsistent extended fall-off arrays in mechanism blob"; return false; }
        xs[xr[k]] = (int)k;
      }
      bool okx = tp.size() == xr.size() + 1 && bp.size() == xr.size() + 1 && pp.size() == bs.size() + 1 &&
                 ty.size() == bs.size() && tp[0] == 0 && bp[0] == 0 && pp[0] == 0 &&
                 (size_t)tp.back() == ts.size() && (size_t)bp.back() == bs.size();
      if (okx && xfo)
        okx = b.F("xfo_kinf").size() == 3 * xr.size() && b.F("xfo_low").size() == 3 * bs.size() &&
              b.F("xfo_tb_eff_m1").size() == ts.size() && (size_t)pp.back() == b.F("xfo_par").size();
      for (size_t k = 0; okx && k + 1 < tp.size(); ++k) okx = tp[k + 1] >= tp[k];
      for (size_t k = 0; okx && k + 1 < bp.size(); ++k) okx = bp[k + 1] > bp[k];
      for (size_t k = 0; okx && k + 1 < pp.size(); ++k) {
        const int np = pp[k + 1] - pp[k];
        okx = (ty[k] == 0 && np == 0) || (ty[k] == 1 && (np == 3 || np == 4)) || (ty[k] == 2 && (np == 3 || np == 5));
      }
      for (size_t k = 0; okx && k < bs.size(); ++k) okx = bs[k] >= -1 && bs[k] < nc;
      for (size_t k = 0; okx && k < ts.size(); ++k) okx = ts[k] >= 0 && ts[k] < nc;
      if (!okx) { err = "inconsistent extended fall-off arrays in mechanism blob"; return false; }
      L.n_xfo = (int)xr.size();
      L.xfo_slot = B.addi(xs);
      L.xfo_tb_ptr = B.addi(tp);
      L.xfo_tb_sp = B.addi(ts.empty() ? none_i : ts);
      L.xfo_bath_ptr = B.addi(bp);
      L.xfo_bath_sp = B.addi(bs.empty() ? none_i : bs);
      L.xfo_type = B.addi(ty.empty() ? none_i : ty);
      L.xfo_par_ptr = B.addi(pp);
    }
    L.cheb_slot = B.addi(cheb_slot);
    L.cheb_rxn = B.addi(cheb_rxn.empty() ? none_i : cheb_rxn);
    L.cheb_nm = B.addi(cheb_nm);
    L.cheb_ptr = B.addi(cheb_ptr);
    L.a_sign = B.addi(b.I("a_sign"));
    L.rev_kind = B.addi(rev_kind);
    L.rev_slot = B.addi(rev_slot);
    L.tb_slot = B.addi(tb_slot);
    L.fo_slot = B.addi(fo_slot);
    L.reac_ptr = B.addi(b.I("reac_ptr"));
    L.reac_sp = B.addi(b.I("reac_species"));
    L.ford_ptr = B.addi(ford_ptr);
    L.ford_sp = B.addi(ford_sp);
    L.prod_ptr = B.addi(b.I("prod_ptr"));
    L.prod_sp = B.addi(b.I("prod_species"));
    L.fr_ptr = B.addi(b.I("fr_ptr"));
    L.fr_rxn = B.addi(b.I("fr_rxn"));
    L.tb_ptr = B.addi(b.I("tb_ptr"));
    L.tb_sp = B.addi(b.I("tb_species"));
    L.fo_type = B.addi(b.I("fo_type"));
    L.fo_single = B.addi(b.I("fo_single"));
    L.fo_ptr = B.addi(b.I("fo_ptr"));
    L.fo_sp = B.addi(b.I("fo_species"));
    {
      std::vector<int> cabr(fr.size() > 0 ? fr.size() : 1, 0);
      if (b.i.count("fo_cabr")) {
        if (b.I("fo_cabr").size() != fr.size()) { err = "inconsistent CABR flags in mechanism blob"; return false; }
        for (size_t k = 0; k < fr.size(); ++k) cabr[k] = b.I("fo_cabr")[k];
      }
      L.fo_cabr = B.addi(cabr);
    }

    L.n_tb = (int)tbr.size();
    L.n_fo = (int)fr.size();
    L.n_rev_th = (int)rth.size();
    L.n_rev_ex = (int)rex.size();
    L.nnz_reac = (int)b.I("reac_species").size();
    L.nnz_prod = (int)b.I("prod_species").size();
    L.nnz_fr = (int)b.I("fr_rxn").size();
    L.nnz_tb = (int)b.I("tb_species").size();
    L.nnz_fo = (int)b.I("fo_species").size();

    // consistency checks (index ranges) so a corrupt blob fails here, not on the device
    auto in_range = [&](const std::vector<int>& v, int lo, int hi) {
      for (int x : v) if (x < lo || x >= hi) return false;
      return true;
    };
    if (!in_range(b.I("reac_species"), 0, nc) || !in_range(b.I("prod_species"), 0, nc) || !in_range(ford_sp, 0, nc) ||
        !in_range(b.I("fr_rxn"), 0, nr) || !in_range(b.I("tb_species"), 0, nc) ||
        !in_range(b.I("fo_species"), 0, nc) || !in_range(tbr, 0, nr) || !in_range(fr, 0, nr)) {
      err = "index out of range in mechanism blob";
      return false;
    }
    // CSR pointer arrays start at 0, never decrease and end at the entry count; value arrays are as long as
    // their index arrays, per-reaction and per-slot arrays as long as the reactions and slots, so that no
    // kernel reads past an array of a corrupt blob
    auto csr_ok = [](const std::vector<int>& ptr, size_t rows, size_t nnz) {
      if (ptr.size() != rows + 1 || ptr[0] != 0 || (size_t)ptr.back() != nnz) return false;
      for (size_t k = 0; k + 1 < ptr.size(); ++k)
        if (ptr[k + 1] < ptr[k]) return false;
      return true;
    };
    const size_t nfo = fr.size();
    bool ok = csr_ok(b.I("reac_ptr"), nr, b.I("reac_species").size()) &&
              csr_ok(b.I("prod_ptr"), nr, b.I("prod_species").size()) && csr_ok(ford_ptr, nr, ford_sp.size()) &&
              csr_ok(b.I("fr_ptr"), nc, b.I("fr_rxn").size()) &&
              csr_ok(b.I("tb_ptr"), tbr.size(), b.I("tb_species").size()) &&
              csr_ok(b.I("fo_ptr"), nfo, b.I("fo_species").size()) &&
              b.F("reac_nu").size() == b.I("reac_species").size() &&
              b.F("prod_nu").size() == b.I("prod_species").size() &&
              b.F("fr_coef").size() == b.I("fr_rxn").size() && b.F("tb_eff_m1").size() == b.I("tb_species").size() &&
              b.F("fo_eff_m1").size() == b.I("fo_species").size() && b.I("fo_type").size() == nfo &&
              b.I("fo_single").size() == nfo && in_range(b.I("fo_type"), 0, 3) &&
              in_range(b.I("fo_single"), -1, nc) && in_range(rth, 0, nr) && in_range(rex, 0, nr);
    for (const char* k : {"beta", "e_over_r", "delta_nu"}) ok = ok && (int)b.F(k).size() == nr;
    for (const char* k : {"fo_lnA", "fo_beta", "fo_e_over_r", "fo_a", "fo_b", "fo_c", "fo_d", "fo_e"})
      ok = ok && b.F(k).size() == nfo;
    for (const char* k : {"lnA_rev", "beta_rev", "e_over_r_rev"}) ok = ok && b.F(k).size() == rex.size();
    for (const char* k : {"cp_lt"}) ok = ok && (int)b.F(k).size() == 5 * nc;
    for (const char* k : {"dh_lt", "ds_ht", "ds_lt"}) ok = ok && (int)b.F(k).size() == 6 * nc;
    ok = ok && (int)b.F("t_mid").size() == nc;
    if (!ok) {
      err = "inconsistent tables in mechanism blob";
      return false;
    }
    if ((int)b.I("reac_ptr").size() != nr + 1 || (int)b.I("prod_ptr").size() != nr + 1 ||
        (int)ford_ptr.size() != nr + 1 || ford_ptr.back() != (int)ford_sp.size() ||
        (ford && b.F("ford_val").size() != ford_sp.size()) ||
        (int)b.I("fr_ptr").size() != nc + 1 || (int)b.F("mw").size() != nc ||
        (int)b.F("cp_ht").size() != 5 * nc || (int)b.F("dh_ht").size() != 6 * nc ||
        (int)b.F("lnA").size() != nr) {
      err = "inconsistent array sizes in mechanism blob";
      return false;
    }
    while (B.d.size() % 2) B.d.push_back(0.);
    while (B.iv.size() % 4) B.iv.push_back(0);
    L.n_double = (int)B.d.size();
    L.n_int = (int)B.iv.size();
    L.bytes = (uint32_t)(B.d.size() * sizeof(double) + B.iv.size() * sizeof(int));
    out.layout = L;
    out.buffer.resize(L.bytes);
    std::memcpy(out.buffer.data(), B.d.data(), B.d.size() * sizeof(double));
    std::memcpy(out.buffer.data() + B.d.size() * sizeof(double), B.iv.data(), B.iv.size() * sizeof(int));
    out.species.clear();
    const auto& nm = b.I("species_names");
    std::string cur;
    for (int ch : nm) {
      if (ch == 0) { out.species.push_back(cur); cur.clear(); }
      else cur.push_back((char)ch);
    }
    out.mw = b.F("mw");
    if (!build_transport(b, nc, out, err)) return false;
  } catch (const std::exception& e) {
    err = e.what();
    return false;
  }
  return true;
}

}  // namespace lsg
