// Project-written stand-in: boost::bind / boost::ref over std::bind / std::ref.
#ifndef PE_ORACLE_SHIM_BIND_HPP
#define PE_ORACLE_SHIM_BIND_HPP
#include <functional>
namespace boost { using std::bind; using std::ref; using std::cref; }
#endif
