// Project-written stand-in: uniform_int over std::uniform_int_distribution.
#ifndef PE_ORACLE_SHIM_UNIFORM_INT_HPP
#define PE_ORACLE_SHIM_UNIFORM_INT_HPP
#include <random>
namespace boost { template <typename T = int> struct uniform_int : std::uniform_int_distribution<T> {
  uniform_int(T a = T(0), T b = T(9)) : std::uniform_int_distribution<T>(a, b) {} }; }
#endif
