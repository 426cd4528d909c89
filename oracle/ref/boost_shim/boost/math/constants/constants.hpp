// Project-written stand-in: the mathematical constants pe takes from Boost.Math, as
// correctly-rounded literals converted to the requested type.
#ifndef PE_ORACLE_SHIM_CONSTANTS_HPP
#define PE_ORACLE_SHIM_CONSTANTS_HPP
namespace boost { namespace math { namespace constants {
template <typename T> inline T pi() { return static_cast<T>(3.14159265358979323846264338327950288L); }
template <typename T> inline T e() { return static_cast<T>(2.71828182845904523536028747135266250L); }
template <typename T> inline T ln_two() { return static_cast<T>(0.693147180559945309417232121458176568L); }
template <typename T> inline T log10_e() { return static_cast<T>(0.434294481903251827651128918916605082L); }
template <typename T> inline T one_div_log10_e() { return static_cast<T>(2.30258509299404568401799145468436421L); }
template <typename T> inline T root_two() { return static_cast<T>(1.41421356237309504880168872420969808L); }
template <typename T> inline T root_three() { return static_cast<T>(1.73205080756887729352744634150587237L); }
}}}
#endif
