// Project-written stand-in: uniform_real over std::uniform_real_distribution.
#ifndef PE_ORACLE_SHIM_UNIFORM_REAL_HPP
#define PE_ORACLE_SHIM_UNIFORM_REAL_HPP
#include <random>
namespace boost { template <typename T = double> struct uniform_real : std::uniform_real_distribution<T> {
  uniform_real(T a = T(0), T b = T(1)) : std::uniform_real_distribution<T>(a, b) {} }; }
#endif
