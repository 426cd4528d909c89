// Project-written stand-in: boost::thread over std::thread.
#ifndef PE_ORACLE_SHIM_THREAD_HPP
#define PE_ORACLE_SHIM_THREAD_HPP
#include <thread>
#include <boost/thread/mutex.hpp>
namespace boost { typedef std::thread thread; }
#endif
