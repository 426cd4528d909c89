// Project-written stand-in: a small printf-style formatter supporting `format(spec) % a % b`.
#ifndef PE_ORACLE_SHIM_FORMAT_HPP
#define PE_ORACLE_SHIM_FORMAT_HPP
#include <cstdio>
#include <sstream>
#include <string>
#include <vector>
#include <ostream>
namespace boost {
class format {
 public:
  explicit format(const std::string& spec) : spec_(spec) {}
  template <typename T> format& operator%(const T& v) { std::ostringstream o; o << v; args_.push_back(o.str()); nums_.push_back(0.0); isnum_.push_back(false); return *this; }
  format& operator%(int v) { return num(v); }
  format& operator%(long v) { return num((double)v); }
  format& operator%(unsigned v) { return num(v); }
  format& operator%(unsigned long v) { return num((double)v); }
  format& operator%(double v) { return num(v); }
  std::string str() const {
    std::string out; size_t a = 0;
    for (size_t i = 0; i < spec_.size(); ++i) {
      if (spec_[i] != '%') { out += spec_[i]; continue; }
      if (i + 1 < spec_.size() && spec_[i + 1] == '%') { out += '%'; ++i; continue; }
      size_t j = i + 1;
      while (j < spec_.size() && std::string("diouxXeEfgGsc").find(spec_[j]) == std::string::npos) ++j;
      std::string f = spec_.substr(i, j - i + 1); char buf[256];
      if (a < args_.size()) {
        char c = spec_[j];
        if (isnum_[a] && std::string("diouxXc").find(c) != std::string::npos) std::snprintf(buf, sizeof buf, f.c_str(), (int)nums_[a]);
        else if (isnum_[a] && c != 's') std::snprintf(buf, sizeof buf, f.c_str(), nums_[a]);
        else std::snprintf(buf, sizeof buf, "%s", args_[a].c_str());
        out += buf; ++a;
      }
      i = j;
    }
    return out;
  }
 private:
  format& num(double v) { std::ostringstream o; o << v; args_.push_back(o.str()); nums_.push_back(v); isnum_.push_back(true); return *this; }
  std::string spec_; std::vector<std::string> args_; std::vector<double> nums_; std::vector<bool> isnum_;
};
inline std::ostream& operator<<(std::ostream& os, const format& f) { return os << f.str(); }
}
#endif
