// Project-written stand-in: boost::hash as an alias of std::hash.
#ifndef PE_ORACLE_SHIM_HASH_HPP
#define PE_ORACLE_SHIM_HASH_HPP
#include <functional>
namespace boost { template <typename T> struct hash : std::hash<T> {}; }
#endif
