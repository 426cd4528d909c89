// Project-written stand-in: exception_ptr helpers over <exception>.
#ifndef PE_ORACLE_SHIM_EXCEPTION_PTR_HPP
#define PE_ORACLE_SHIM_EXCEPTION_PTR_HPP
#include <exception>
namespace boost {
using std::exception_ptr; using std::current_exception; using std::rethrow_exception;
template <typename T> inline const T& enable_current_exception(const T& t) { return t; }
}
#endif
