// Project-written stand-in (maps to <type_traits>); see boost/type_traits.hpp.
#include <boost/type_traits.hpp>
