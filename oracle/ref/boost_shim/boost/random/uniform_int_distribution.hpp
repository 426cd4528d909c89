// Project-written stand-in: boost::random::uniform_int_distribution over <random>.
#ifndef PE_ORACLE_SHIM_UNIFORM_INT_DIST_HPP
#define PE_ORACLE_SHIM_UNIFORM_INT_DIST_HPP
#include <random>
namespace boost { namespace random { using std::uniform_int_distribution; } }
#endif
