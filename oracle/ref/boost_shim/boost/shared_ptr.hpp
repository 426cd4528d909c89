// Project-written stand-in: boost::shared_ptr mapped to std::shared_ptr.
#ifndef PE_ORACLE_SHIM_SHARED_PTR_HPP
#define PE_ORACLE_SHIM_SHARED_PTR_HPP
#include <memory>
namespace boost { using std::shared_ptr; using std::dynamic_pointer_cast; using std::static_pointer_cast; }
#endif
