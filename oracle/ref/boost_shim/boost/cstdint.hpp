// Project-written stand-in: fixed-width integers from <cstdint>.
#ifndef PE_ORACLE_SHIM_CSTDINT_HPP
#define PE_ORACLE_SHIM_CSTDINT_HPP
#include <cstdint>
namespace boost { using std::int8_t; using std::int16_t; using std::int32_t; using std::int64_t;
using std::uint8_t; using std::uint16_t; using std::uint32_t; using std::uint64_t; }
#endif
