// Project-written stand-in: boost::unordered_map over std::unordered_map.
#ifndef PE_ORACLE_SHIM_UNORDERED_MAP_HPP
#define PE_ORACLE_SHIM_UNORDERED_MAP_HPP
#include <unordered_map>
namespace boost { using std::unordered_map; }
#endif
