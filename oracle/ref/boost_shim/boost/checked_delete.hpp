// Project-written stand-in: checked_delete / checked_array_delete.
#ifndef PE_ORACLE_SHIM_CHECKED_DELETE_HPP
#define PE_ORACLE_SHIM_CHECKED_DELETE_HPP
namespace boost {
template <typename T> inline void checked_delete(T* p) { typedef char complete[sizeof(T) ? 1 : -1]; (void)sizeof(complete); delete p; }
template <typename T> inline void checked_array_delete(T* p) { typedef char complete[sizeof(T) ? 1 : -1]; (void)sizeof(complete); delete[] p; }
}
#endif
