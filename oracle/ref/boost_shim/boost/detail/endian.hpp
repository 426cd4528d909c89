// Project-written stand-in: byte-order macro from the compiler's predefined macros.
#ifndef PE_ORACLE_SHIM_ENDIAN_HPP
#define PE_ORACLE_SHIM_ENDIAN_HPP
#if defined(__BYTE_ORDER__) && __BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__
#define BOOST_LITTLE_ENDIAN
#else
#define BOOST_BIG_ENDIAN
#endif
#endif
