// TEST INFRASTRUCTURE ONLY: stands in for the reference's
// math/OpenSMOKEUtilities.h (which pulls in Boost.Filesystem and RapidXML,
// both absent here) when the reference's dense ODE solver templates are
// compiled for the oracle cross-check.  It supplies the few helpers those
// templates call, each restated from the reference's definition:
//   MachEps / MachEpsFloat            math/OpenSMOKEFunctions.hpp:60-87
//   OPENSMOKE_MACH_EPS_*              math/OpenSMOKEFunctions.hpp:39-40
//   ErrorControl                      math/OpenSMOKEUtilities.hpp:689-701
//   Abs, MaxAbs                       math/OpenSMOKEUtilities.hpp (templates)
//   OpenSMOKEGetCpuTime               math/OpenSMOKEFunctions.hpp:193-200 (timing only)
//   ErrorMessage                      math/OpenSMOKEFunctions.hpp:42-49, which
//                                     waits for a key and exits; here it throws
// The constants and enums come from the reference's own
// math/OpenSMOKEStdInclude.h.
#ifndef LSG_REFPIN_OPENSMOKE_UTILITIES
#define LSG_REFPIN_OPENSMOKE_UTILITIES

#include <cmath>
#include <ctime>
#include <stdexcept>
#include <string>

#include "math/OpenSMOKEStdInclude.h"
#include "boost/lexical_cast.hpp"

namespace OpenSMOKE {

inline float MachEpsFloat() {
  float macheps = 1.F, eps = 2.F;
  while (eps != 1.F) {
    macheps /= 2.F;
    eps = float(1.F + macheps);
  }
  return macheps < 1.e-7 ? 1.192092896e-07F : macheps * 2.F;
}

inline double MachEps() {
  double macheps = 1., eps = 2.;
  while (eps != 1.) {
    macheps /= 2.;
    eps = 1. + macheps;
  }
  return macheps * 2.;
}

static const float OPENSMOKE_MACH_EPS_FLOAT = MachEpsFloat();
static const double OPENSMOKE_MACH_EPS_DOUBLE = MachEps();

inline double OpenSMOKEGetCpuTime() { return (double)std::clock() / CLOCKS_PER_SEC; }

inline void ErrorMessage(const std::string where, const std::string what) {
  throw std::runtime_error(where + ": " + what);
}

template <typename T>
inline T Abs(T const& a) { return a < 0 ? -a : a; }

template <typename T>
inline T MaxAbs(T const& a, T const& b) { return Abs(a) > Abs(b) ? Abs(a) : Abs(b); }

template <typename T>
double ErrorControl(const T& w, const T& e) {
  const std::size_t ne = w.size();
  double sum = 0.;
  for (unsigned int i = 0; i < ne; i++) {
    const double coeff = w(i) * e(i);
    sum += coeff * coeff;
  }
  return std::sqrt(sum / double(ne));
}

}  // namespace OpenSMOKE

#endif
