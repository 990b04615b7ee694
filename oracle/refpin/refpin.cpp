// TEST INFRASTRUCTURE ONLY: the reference's own integrator driving the
// oracle's right-hand side.
//
// The reference's dense BDF integrator -- the class templates
// OdeSMOKE::MultiValueSolver< MethodGear< KernelDense<System> > > of
// solvers/openSMOKEpp4laminarSMOKE/math/native-ode-solvers/
// {MultiValueSolver,MethodGear,KernelDense,OdeSolverUtilities}.{h,hpp} --
// is compiled here unchanged, from the reference's files, against small
// stand-ins for Eigen and the two OpenSMOKE/Boost helpers it calls
// (oracle/refpin/shim).  System is the adaptor below: it plays the role of
// BatchReactorHomogeneousConstantPressure_ODE_OpenSMOKE and evaluates the
// oracle's restatement of BatchReactorHomogeneousConstantPressure::Equations.
// The per-cell driver below makes the calls of
// solvers/laminarSMOKE/unsteady/chemistry_DI.H:92-169 in its order
// (SetInitialConditions, SetFullPivoting, tolerances, SetMinimumValues,
// SetMaximumValues, Solve, Solution, QR), with the clipping and
// renormalisation of :100-129 and utilities.H:153-200.
//
// Used by tests/test_refpin.py to pin the oracle's integrator (oracle.cpp,
// class Gear) to the reference's code: on the same cells both must agree bit
// for bit, counters included.  Built by oracle/refpin/Makefile into
// oracle/_ref/ only where the reference sources are present.
#include "../oracle.cpp"

#include "MultiValueSolver.h"
#include "MethodGear.h"
#include "KernelDense.h"

namespace refpin {

// The ODE-system adaptor the reference's KernelDense derives from
// (the role of solvers/laminarSMOKE/unsteady/ODESystemVirtualClassWithOpenSMOKEVectors.H).
class ReactorSystem {
 public:
  void SetReactor(orc::Reactor* r) { reactor_ = r; }
  long long equations_calls() const { return calls_; }

 protected:
  unsigned int ne_ = 0;
  void MemoryAllocation() {}
  void Equations(const Eigen::VectorXd& y, const double /*t*/, Eigen::VectorXd& dy) {
    reactor_->equations(y.data(), dy.data());
    ++calls_;
  }
  void Jacobian(const Eigen::VectorXd&, const double, Eigen::MatrixXd&) {}
  void Print(const double, const Eigen::VectorXd&) {}

 private:
  orc::Reactor* reactor_ = nullptr;
  long long calls_ = 0;
};

typedef OdeSMOKE::KernelDense<ReactorSystem> DenseKernel;
typedef OdeSMOKE::MethodGear<DenseKernel> Gear;
typedef OdeSMOKE::MultiValueSolver<Gear> Solver;

}  // namespace refpin

extern "C" {

// Same arguments and outputs as orc_reaction_step (constant-pressure reactor,
// a fresh solver object per cell, i.e. sequential_state 0).
int ref_reaction_step(void* mech, const orc_options* o, int ncells, double* Y, double* T, double p, double t0,
                      const double* dt, double dt_scalar, double* Q, int* status, long long* counters,
                      int nthreads) {
  const orc::Mech& m = *(const orc::Mech*)mech;
  const int NC = m.nc;
  const unsigned NEQ = NC + 1;
  int nerr = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel reduction(+ : nerr)
  {
    orc::Reactor reactor(m);
    Eigen::VectorXd yMin(NEQ), yMax(NEQ), y0(NEQ), yf(NEQ);
    for (unsigned i = 0; i < NEQ; ++i) { yMin(i) = 0.; yMax(i) = 1.; }
    yMin(NC) = o->y_min_T;
    yMax(NC) = o->y_max_T;
#pragma omp for schedule(dynamic, 1)
    for (int cell = 0; cell < ncells; ++cell) {
      double* Yc = Y + (size_t)cell * NC;
      int st = 0;
      long long cnt[orc::NCOUNT] = {};
      if (T[cell] > o->tmin_chem) {
        for (int i = 0; i < NC; ++i) y0(i) = Yc[i];
        y0(NC) = T[cell];
        double sum = 0.;
        for (int i = 0; i < NC; ++i) {
          if (y0(i) < 0.) y0(i) = 0.;
          sum += y0(i);
        }
        for (int i = 0; i < NC; ++i) y0(i) /= sum;
        reactor.P0 = p;
        reactor.rho0 = 0.;
        reactor.energy = o->energy != 0;
        if (!reactor.energy) reactor.QR = 0.;
        refpin::Solver solver;
        solver.SetReactor(&reactor);
        solver.SetInitialConditions(t0, y0);
        solver.SetFullPivoting(o->full_pivoting != 0);
        solver.SetAbsoluteTolerances(o->atol);
        solver.SetRelativeTolerances(o->rtol);
        solver.SetMinimumValues(yMin);
        solver.SetMaximumValues(yMax);
        solver.SetMaximumNumberOfSteps((unsigned)o->max_steps);
        const double dtc = dt ? dt[cell] : dt_scalar;
        st = (int)solver.Solve(t0 + dtc);
        solver.Solution(yf);
        if (Q) Q[cell] = reactor.QR;
        cnt[orc::COUNT_STEPS] = solver.numberOfSteps();
        cnt[orc::COUNT_JAC_RHS] = solver.numberOfFunctionCallsForJacobian();
        cnt[orc::COUNT_RHS] = solver.equations_calls() - cnt[orc::COUNT_JAC_RHS];
        cnt[orc::COUNT_JAC] = solver.numberOfJacobianEvaluations();
        cnt[orc::COUNT_FACT] = solver.numberOfMatrixFactorizations();
        cnt[orc::COUNT_SOLVE] = solver.numberOfLinearSystemSolutions();
        cnt[orc::COUNT_ERRFAIL] = solver.numberOfErrorCheckFailure();
        cnt[orc::COUNT_CONVFAIL] = solver.numberOfConvergenceFailure();
        if (st < 0) nerr++;
      } else {
        for (int i = 0; i < NC; ++i) yf(i) = Yc[i];
        yf(NC) = T[cell];
      }
      if (counters)
        for (int k = 0; k < orc::NCOUNT; ++k) counters[(size_t)cell * orc::NCOUNT + k] = cnt[k];
      double s = 0.;
      for (int i = 0; i < NC; ++i) s += yf(i);
      for (int i = 0; i < NC; ++i) Yc[i] = yf(i) / s;
      if (o->energy) T[cell] = yf(NC);
      if (status) status[cell] = st;
    }
  }
  return nerr;
}

}  // extern "C"
