// Project-written stand-in for the parts of Boost.TypeTraits that pe uses, mapped to <type_traits>.
// Used only to compile the reference as a test oracle.  No Boost source is copied.
#ifndef PE_ORACLE_SHIM_TYPE_TRAITS_HPP
#define PE_ORACLE_SHIM_TYPE_TRAITS_HPP
#include <type_traits>
#include <cstddef>
namespace boost {
using std::integral_constant; using std::true_type; using std::false_type;
using std::is_base_of; using std::remove_reference; using std::remove_cv; using std::is_void;
using std::is_volatile; using std::is_unsigned; using std::is_signed; using std::is_reference;
using std::is_pointer; using std::is_pod; using std::is_object; using std::is_integral;
using std::is_fundamental; using std::is_floating_point; using std::is_convertible;
using std::is_const; using std::is_class; using std::is_arithmetic;
template <typename F> struct function_traits;
template <typename R, typename... A> struct function_traits<R(A...)> {
  static const std::size_t arity = sizeof...(A);
  typedef R result_type;
};
}
#endif
