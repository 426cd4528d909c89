// Project-written stand-in: boost::result_of over std::result_of.
#ifndef PE_ORACLE_SHIM_RESULT_OF_HPP
#define PE_ORACLE_SHIM_RESULT_OF_HPP
#include <type_traits>
namespace boost { using std::result_of; }
#endif
