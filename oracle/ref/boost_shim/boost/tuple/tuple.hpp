// Project-written stand-in: boost::tuple / make_tuple / get over <tuple>.
#ifndef PE_ORACLE_SHIM_TUPLE_HPP
#define PE_ORACLE_SHIM_TUPLE_HPP
#include <tuple>
namespace boost { using std::tuple; using std::make_tuple; using std::get; }
#endif
