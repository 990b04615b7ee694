// TEST INFRASTRUCTURE ONLY: the one Boost facility the reference's dense ODE
// solver templates use (boost::lexical_cast<unsigned int> of a vector size,
// MultiValueSolver.hpp:383), for the oracle cross-check; Boost is absent here.
#ifndef LSG_REFPIN_BOOST_LEXICAL_CAST
#define LSG_REFPIN_BOOST_LEXICAL_CAST
namespace boost {
template <typename To, typename From>
inline To lexical_cast(const From& v) { return static_cast<To>(v); }
}  // namespace boost
#endif
