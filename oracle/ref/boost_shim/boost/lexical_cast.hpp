// Project-written stand-in: lexical_cast through a stringstream.
#ifndef PE_ORACLE_SHIM_LEXICAL_CAST_HPP
#define PE_ORACLE_SHIM_LEXICAL_CAST_HPP
#include <sstream>
#include <string>
#include <stdexcept>
namespace boost {
struct bad_lexical_cast : std::bad_cast {};
template <typename T, typename S> inline T lexical_cast(const S& s) {
  std::stringstream ss; ss << s; T t; if (!(ss >> t)) throw bad_lexical_cast(); return t; }
template <> inline std::string lexical_cast<std::string, std::string>(const std::string& s) { return s; }
}
#endif
