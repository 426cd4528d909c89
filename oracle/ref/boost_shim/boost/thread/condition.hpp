// Project-written stand-in: boost::condition_variable over std::condition_variable_any.
#ifndef PE_ORACLE_SHIM_CONDITION_HPP
#define PE_ORACLE_SHIM_CONDITION_HPP
#include <condition_variable>
#include <boost/thread/mutex.hpp>
namespace boost { typedef std::condition_variable_any condition_variable; typedef std::condition_variable_any condition; }
#endif
