// Project-written stand-in: mt19937 from <random>.
#ifndef PE_ORACLE_SHIM_MT_HPP
#define PE_ORACLE_SHIM_MT_HPP
#include <random>
namespace boost { typedef std::mt19937 mt19937; namespace random { typedef std::mt19937 mt19937; } }
#endif
