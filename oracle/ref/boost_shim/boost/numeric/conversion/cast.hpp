// Project-written stand-in: numeric_cast as a plain static_cast (no range check).
#ifndef PE_ORACLE_SHIM_NUMERIC_CAST_HPP
#define PE_ORACLE_SHIM_NUMERIC_CAST_HPP
namespace boost { template <typename T, typename S> inline T numeric_cast(S s) { return static_cast<T>(s); } }
#endif
