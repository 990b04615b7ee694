/* C++ layer over the C ABI of lsmoke_gpu.h with the names and call order of
 * the reference's chemistry loop (solvers/laminarSMOKE/unsteady/
 * chemistry_DI.H:131-167), batched over a whole cell field:
 *
 *   reference (per cell)                                here (per field)
 *   batchReactor.SetReactor(P)                          reactor.SetReactor(P)
 *   batchReactor.SetEnergyEquation(on)                  reactor.SetEnergyEquation(on)
 *   odeSolver().SetInitialConditions(t0, y0)            solver.SetInitialConditions(t0, ncells, Y, T)
 *   odeSolver().SetFullPivoting(false)                  solver.SetFullPivoting(false)
 *   odeSolver().SetAbsoluteTolerances(atol)             solver.SetAbsoluteTolerances(atol)
 *   odeSolver().SetRelativeTolerances(rtol)             solver.SetRelativeTolerances(rtol)
 *   odeSolver().SetMinimumValues(yMin)                  solver.SetMinimumValues(yMin)   (yMin[NC] = T bound)
 *   odeSolver().SetMaximumValues(yMax)                  solver.SetMaximumValues(yMax)
 *   status = odeSolver().Solve(t0 + dt)                 statuses = solver.Solve(t0 + dt) or Solve(dt[])
 *   odeSolver().Solution(yf)                            the Y, T arrays given to SetInitialConditions
 *   Q = batchReactor.QR()                               solver.QR()[cell]
 *
 * (BatchReactorHomogeneousConstantPressure.H:60-141, MultiValueSolver.hpp:
 * 367-617.)  As the driver loop does around those calls, the step clips
 * negative mass fractions and renormalises before the solve and renormalises
 * after it (chemistry_DI.H:100-129, 219).  Errors the reference reports by
 * printing or exiting throw lsmoke::Error, which carries the C-ABI code.
 * Header-only; link with liblsmoke_gpu.so. */
#ifndef LSMOKE_GPU_HPP
#define LSMOKE_GPU_HPP

#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "lsmoke_gpu.h"

namespace lsmoke {

/* OdeSolverUtilities.h:83-97 */
enum OdeStatus {
  ODE_STATUS_TO_BE_INITIALIZED = 1,
  ODE_STATUS_CONTINUATION = 2,
  ODE_STATUS_STOP_INTEGRATION_FOR_SMALL_YPRIME_NORM1 = 3,
  ODE_STATUS_MAX_NUMBER_OF_STEPS_REACHED = -1,
  ODE_STATUS_TOO_STRICT_TOLERANCES = -2,
  ODE_STATUS_ILLEGAL_CONTINUATION_REQUEST = -3,
  ODE_STATUS_MAX_NUMBER_ERRORTEST_FAILURES = -4,
  ODE_STATUS_MAX_NUMBER_CONVERGENCETEST_FAILURES = -5,
  ODE_STATUS_TOO_SMALL_STEP_SIZE = -6,
  ODE_STATUS_ILLEGAL_MAX_INDEPENDENT_VARIABLE = -7,
  ODE_STATUS_ILLEGAL_CONSTRAINTS = -9,
  ODE_STATUS_EXCEPTION_HANDLING_STOP = -10,
  ODE_STATUS_YOU_CANNOT_OVERSHOOT_TCRITIC = -12
};

class Error : public std::runtime_error {
 public:
  Error(const std::string& what, int code)
      : std::runtime_error(what + ": " + lsg_strerror(code) + " (" + std::to_string(code) + ")"), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

inline void check(int rc, const char* what) {
  if (rc != LSG_OK) throw Error(what, rc);
}

/* A mechanism blob already in host memory. */
struct Blob {
  const void* data;
  size_t size;
};

/* Device-resident mechanism (the kinetics.xml the reference reads). */
class Mechanism {
 public:
  explicit Mechanism(const std::string& path, int device = 0) : device_(device) {
    check(lsg_mech_load_file(path.c_str(), device, &m_), "lsg_mech_load_file");
    check(lsg_mech_info(m_, &ns_, &nr_), "lsg_mech_info");
  }
  explicit Mechanism(Blob blob, int device = 0) : device_(device) {
    check(lsg_mech_load_blob(blob.data, blob.size, device, &m_), "lsg_mech_load_blob");
    check(lsg_mech_info(m_, &ns_, &nr_), "lsg_mech_info");
  }
  ~Mechanism() { if (m_) lsg_mech_destroy(m_); }
  Mechanism(const Mechanism&) = delete;
  Mechanism& operator=(const Mechanism&) = delete;
  int NumberOfSpecies() const { return ns_; }
  int NumberOfReactions() const { return nr_; }
  const lsg_mech* get() const { return m_; }
  int device() const { return device_; }

 private:
  lsg_mech* m_ = nullptr;
  int device_ = 0;
  int ns_ = 0, nr_ = 0;
};

/* The reactor settings every cell of a call shares. */
/* The DRG settings of the reference's DRG dictionary (solvers/laminarSMOKE/unsteady/chemistry_DRG.H with
 * DRG.hpp): key species indices, (temperature, epsilon) bands, the minimum temperature.  Set on the reactor
 * with SetDRG, as the reference does; the solver then runs the DRG-reduced step over the field and the
 * important species / reactions of each cell are read back here. */
class DRG {
 public:
  explicit DRG(std::vector<int> key_species) : key_(std::move(key_species)) {
    if (key_.empty()) throw Error("DRG: no key species", LSG_ERR_ARG);
  }
  /* A cell takes the epsilon of the first band whose temperature is above its own. */
  void SetTemperatureBands(const std::vector<double>& T, const std::vector<double>& epsilon) {
    if (T.empty() || T.size() != epsilon.size() || T.size() > LSG_DRG_MAX_BANDS)
      throw Error("DRG::SetTemperatureBands", LSG_ERR_ARG);
    band_T_ = T;
    band_eps_ = epsilon;
  }
  void SetEpsilon(double epsilon0) { eps0_ = epsilon0; }
  void SetMinimumTemperature(double T) { min_T_ = T; }
  /* true (the reference's behaviour): the solver options reach the first cell only. */
  void SetOptionsOnFirstCellOnly(bool flag) { first_only_ = flag; }
  const std::vector<int>& NumberOfImportantSpecies() const { return n_species_; }
  const std::vector<int>& NumberOfImportantReactions() const { return n_reactions_; }

  lsg_drg_options options() const {
    lsg_drg_options o{};
    o.key = key_.data();
    o.nkey = (int)key_.size();
    o.band_T = band_T_.data();
    o.band_eps = band_eps_.data();
    o.nbands = (int)band_T_.size();
    o.epsilon0 = eps0_;
    o.min_T = min_T_;
    o.first_cell_options_only = first_only_ ? 1 : 0;
    return o;
  }
  std::vector<int>& n_species() { return n_species_; }
  std::vector<int>& n_reactions() { return n_reactions_; }

 private:
  std::vector<int> key_;
  std::vector<double> band_T_{1.e6}, band_eps_{1.e-2};
  double eps0_ = 1.e-2;
  double min_T_ = 300.;
  bool first_only_ = true;
  std::vector<int> n_species_, n_reactions_;
};

class BatchReactorHomogeneousConstantPressure {
 public:
  /* The reduced system of chemistry_DRG.H (nullptr: the full reactor). */
  void SetDRG(DRG* drg) { drg_ = drg; }
  DRG* drg() const { return drg_; }
  void SetReactor(double P0) {
    if (!(P0 > 0.)) throw Error("SetReactor", LSG_ERR_ARG);
    P0_ = P0;
  }
  void SetEnergyEquation(bool flag) { energy_ = flag; }
  double P0() const { return P0_; }
  bool energy() const { return energy_; }

 private:
  double P0_ = 101325.;
  bool energy_ = true;
  DRG* drg_ = nullptr;
};

/* One context: the batched counterpart of the reference's solver object. */
class MultiValueSolver {
 public:
  MultiValueSolver(const Mechanism& mech, const BatchReactorHomogeneousConstantPressure& reactor,
                   int precision = LSG_PRECISION_FP64)
      : mech_(mech), reactor_(reactor) {
    lsg_options_default(&opt_);
    opt_.precision = precision;
    check(lsg_ctx_create(mech.get(), &opt_, mech.device(), &ctx_), "lsg_ctx_create");
  }
  ~MultiValueSolver() { if (ctx_) lsg_ctx_destroy(ctx_); }
  MultiValueSolver(const MultiValueSolver&) = delete;
  MultiValueSolver& operator=(const MultiValueSolver&) = delete;

  /* Y_species: NC pointers to ncells mass fractions each (the OpenFOAM field
   * layout), T: ncells temperatures.  Both are read by Solve and receive the
   * solution in place. */
  void SetInitialConditions(double t0, int ncells, double* const* Y_species, double* T) {
    if (ncells < 0 || !Y_species || !T) throw Error("SetInitialConditions", LSG_ERR_ARG);
    t0_ = t0;
    n_ = ncells;
    Y_ = Y_species;
    T_ = T;
  }
  /* Only partial pivoting, the reference's default, is implemented. */
  void SetFullPivoting(bool flag) {
    if (flag) throw Error("SetFullPivoting", LSG_ERR_UNSUPPORTED);
  }
  void SetAbsoluteTolerances(double atol) { opt_.atol = atol; dirty_ = true; }
  void SetRelativeTolerances(double rtol) { opt_.rtol = rtol; dirty_ = true; }
  /* yMin / yMax as chemistry_DI.H:82-83 builds them: [0, 1] for every mass
   * fraction (the only bounds supported) and the T bounds in the last entry. */
  void SetMinimumValues(const std::vector<double>& yMin) {
    bounds(yMin, 0., "SetMinimumValues");
    opt_.y_min_T = yMin.back();
    dirty_ = true;
  }
  void SetMaximumValues(const std::vector<double>& yMax) {
    bounds(yMax, 1., "SetMaximumValues");
    opt_.y_max_T = yMax.back();
    dirty_ = true;
  }
  /* minTemperature4Chemistry: cells at or below it are only renormalised. */
  void SetMinimumTemperatureForChemistry(double tmin) { opt_.tmin_chem = tmin; dirty_ = true; }

  /* Integrates every cell from t0 to tOut.  Returns the OdeStatus of each cell. */
  const std::vector<int>& Solve(double tOut) { return solve(nullptr, tOut - t0_); }
  /* Local time stepping: cell i integrates from t0 to t0 + dt[i]. */
  const std::vector<int>& Solve(const double* dt) { return solve(dt, 0.); }

  const std::vector<double>& QR() const { return Q_; }
  const std::vector<int>& NumberOfSteps() const { return nsteps_; }
  lsg_ctx* context() { return ctx_; }

 private:
  void apply() {   // the reactor's energy switch and changed solver settings, pushed to the context
    const int e = reactor_.energy() ? 1 : 0;
    if (opt_.energy != e) {
      opt_.energy = e;
      dirty_ = true;
    }
    if (dirty_) {
      check(lsg_ctx_set_options(ctx_, &opt_), "lsg_ctx_set_options");
      dirty_ = false;
    }
  }
  void bounds(const std::vector<double>& v, double species_value, const char* what) {
    if ((int)v.size() != mech_.NumberOfSpecies() + 1) throw Error(what, LSG_ERR_ARG);
    for (size_t i = 0; i + 1 < v.size(); ++i)
      if (v[i] != species_value) throw Error(what, LSG_ERR_UNSUPPORTED);
  }
  const std::vector<int>& solve(const double* dt, double dt_scalar) {
    if (!Y_ && n_ > 0) throw Error("Solve before SetInitialConditions", LSG_ERR_ARG);
    apply();
    status_.assign(n_, 0);
    nsteps_.assign(n_, 0);
    Q_.assign(n_, 0.);
    if (DRG* drg = reactor_.drg()) {   // chemistry_DRG.H: the reduced step of every cell
      const lsg_drg_options o = drg->options();
      drg->n_species().assign(n_, 0);
      drg->n_reactions().assign(n_, 0);
      check(lsg_reaction_step_drg(ctx_, n_, mech_.NumberOfSpecies(), Y_, T_, reactor_.P0(), t0_, dt, dt_scalar, &o,
                                  Q_.data(), status_.data(), drg->n_species().data(), drg->n_reactions().data()),
            "lsg_reaction_step_drg");
      return status_;
    }
    check(lsg_reaction_step(ctx_, n_, mech_.NumberOfSpecies(), Y_, T_, reactor_.P0(), t0_, dt, dt_scalar,
                            Q_.data(), status_.data(), nsteps_.data()),
          "lsg_reaction_step");
    return status_;
  }

  const Mechanism& mech_;
  const BatchReactorHomogeneousConstantPressure& reactor_;
  lsg_options opt_{};
  bool dirty_ = false;
  lsg_ctx* ctx_ = nullptr;
  double t0_ = 0.;
  int n_ = 0;
  double* const* Y_ = nullptr;
  double* T_ = nullptr;
  std::vector<int> status_, nsteps_;
  std::vector<double> Q_;
};

/* The property update after the step (solvers/laminarSMOKE/properties.H:40-190) over a whole field, in one
 * call: what the reference gets per cell from ThermodynamicsMap_CHEMKIN (MoleFractions_From_MassFractions,
 * hMolar_Mixture_From_MoleFractions, cpMolar_Mixture_From_MoleFractions, cpMolar_Species) and
 * TransportPropertiesMap_CHEMKIN (DynamicViscosity, ThermalConductivity, MassDiffusionCoefficients,
 * ThermalDiffusionRatios).  Needs a mechanism compiled with its transport file. */
class TransportPropertiesMap {
 public:
  /* Host fields, resized by Evaluate; species fields species-major [NC][ncells], Dsoret
   * [ThermalDiffusionSpecies().size()][ncells]. */
  struct Fields {
    std::vector<double> X, cTot, psi, mu, lambda, cp, cv, h, MWmix, cp_species, Dmix, Dsoret;
  };

  explicit TransportPropertiesMap(const Mechanism& mech) : mech_(mech) {
    int has = 0, nt = 0;
    iteta_.assign(mech.NumberOfSpecies(), 0);
    check(lsg_mech_transport_info(mech.get(), &has, &nt, iteta_.data()), "lsg_mech_transport_info");
    if (!has) throw Error("TransportPropertiesMap: the mechanism has no transport data", LSG_ERR_UNSUPPORTED);
    iteta_.resize(nt);
    lsg_options o;
    lsg_options_default(&o);
    check(lsg_ctx_create(mech.get(), &o, mech.device(), &ctx_), "lsg_ctx_create");
  }
  ~TransportPropertiesMap() { if (ctx_) lsg_ctx_destroy(ctx_); }
  TransportPropertiesMap(const TransportPropertiesMap&) = delete;
  TransportPropertiesMap& operator=(const TransportPropertiesMap&) = delete;

  /* energyEquation: lambda, cp, cv and the species cp are evaluated. */
  void SetEnergyEquation(bool flag) { energy_ = flag; }
  /* simplifiedTransportProperties: mu = 1.8405e-5 (T/300)^0.6759, lambda = mu cp / 0.7. */
  void SetSimplifiedTransportProperties(bool flag) { simplified_ = flag; }
  /* DIFFUSIVITY_MODEL_LEWIS_NUMBERS with one Lewis number per species; an empty vector selects the
   * mixture-averaged coefficients (DIFFUSIVITY_MODEL_MULTICOMPONENT). */
  void SetLewisNumbers(const std::vector<double>& le) {
    if (!le.empty() && (int)le.size() != mech_.NumberOfSpecies()) throw Error("SetLewisNumbers", LSG_ERR_ARG);
    lewis_ = le;
  }
  /* soretEffect: thermal-diffusion terms of the light species. */
  void SetSoretEffect(bool flag) { soret_ = flag; }
  /* Species with thermal-diffusion ratios (iThermalDiffusionRatios, 0-based). */
  const std::vector<int>& ThermalDiffusionSpecies() const { return iteta_; }

  /* Y [NC][ncells] mass fractions, T [ncells], p [ncells] (or nullptr and p_scalar). */
  void Evaluate(int ncells, const double* Y, const double* T, const double* p, Fields& f, double p_scalar = 0.) {
    if (ncells < 0 || !Y || !T) throw Error("Evaluate", LSG_ERR_ARG);
    const size_t n = (size_t)ncells, nc = (size_t)mech_.NumberOfSpecies();
    const bool thermal = energy_ || !lewis_.empty();
    f.X.resize(nc * n);
    f.cTot.resize(n);
    f.psi.resize(n);
    f.mu.resize(n);
    f.h.resize(n);
    f.MWmix.resize(n);
    f.Dmix.resize(nc * n);
    f.lambda.resize(thermal ? n : 0);
    f.cp.resize(thermal ? n : 0);
    f.cv.resize(thermal ? n : 0);
    f.cp_species.resize(thermal ? nc * n : 0);
    f.Dsoret.resize(soret_ ? iteta_.size() * n : 0);
    auto ptr = [](std::vector<double>& v) { return v.empty() ? nullptr : v.data(); };
    lsg_property_fields pf = {ptr(f.X),  ptr(f.cTot), ptr(f.psi), ptr(f.mu),    ptr(f.lambda),     ptr(f.cp),
                              ptr(f.cv), ptr(f.h),    ptr(f.MWmix), ptr(f.cp_species), ptr(f.Dmix), nullptr};
    if (soret_ && !iteta_.empty()) pf.Dsoret = f.Dsoret.data();
    lsg_property_options po = {energy_ ? 1 : 0, simplified_ ? 1 : 0, lewis_.empty() ? nullptr : lewis_.data()};
    check(lsg_properties(ctx_, ncells, (int)nc, Y, T, p, p_scalar, &po, &pf), "lsg_properties");
  }

 private:
  const Mechanism& mech_;
  lsg_ctx* ctx_ = nullptr;
  std::vector<int> iteta_;
  std::vector<double> lewis_;
  bool energy_ = true, simplified_ = false, soret_ = false;
};

}  // namespace lsmoke

#endif /* LSMOKE_GPU_HPP */
