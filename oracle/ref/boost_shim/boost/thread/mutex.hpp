// Project-written stand-in: boost::mutex with a scoped_lock typedef, over std::mutex.
#ifndef PE_ORACLE_SHIM_MUTEX_HPP
#define PE_ORACLE_SHIM_MUTEX_HPP
#include <mutex>
namespace boost {
struct mutex : std::mutex { typedef std::unique_lock<std::mutex> scoped_lock; };
}
#endif
