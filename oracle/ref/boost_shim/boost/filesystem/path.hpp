// Project-written stand-in: a string-backed filesystem::path with the few members pe uses.
#ifndef PE_ORACLE_SHIM_FS_PATH_HPP
#define PE_ORACLE_SHIM_FS_PATH_HPP
#include <string>
#include <ostream>
namespace boost { namespace filesystem {
class path {
 public:
  path() {}
  path(const std::string& s) : s_(s) {}
  path(const char* s) : s_(s) {}
  const std::string& string() const { return s_; }
  const char* c_str() const { return s_.c_str(); }
  bool empty() const { return s_.empty(); }
  path& operator/=(const path& p) { if (!s_.empty() && s_[s_.size()-1] != '/') s_ += '/'; s_ += p.s_; return *this; }
  path filename() const { std::string::size_type k = s_.rfind('/'); return k == std::string::npos ? *this : path(s_.substr(k + 1)); }
  path parent_path() const { std::string::size_type k = s_.rfind('/'); return k == std::string::npos ? path() : path(s_.substr(0, k)); }
  std::string extension() const { std::string f = filename().s_; std::string::size_type k = f.rfind('.'); return k == std::string::npos ? std::string() : f.substr(k); }
  std::string stem() const { std::string f = filename().s_; std::string::size_type k = f.rfind('.'); return k == std::string::npos ? f : f.substr(0, k); }
  path& replace_extension(const std::string& e) { std::string::size_type k = s_.rfind('.'); if (k != std::string::npos && s_.find('/', k) == std::string::npos) s_.erase(k); s_ += e; return *this; }
 private:
  std::string s_;
};
inline path operator/(const path& a, const path& b) { path r(a); r /= b; return r; }
inline std::ostream& operator<<(std::ostream& os, const path& p) { return os << '"' << p.string() << '"'; }
}}
#endif
