// Project-written stand-in: the filesystem operations pe uses, over POSIX calls.
#ifndef PE_ORACLE_SHIM_FS_OPS_HPP
#define PE_ORACLE_SHIM_FS_OPS_HPP
#include <boost/filesystem/path.hpp>
#include <sys/stat.h>
#include <sys/types.h>
namespace boost { namespace filesystem {
inline bool exists(const path& p) { struct stat st; return ::stat(p.c_str(), &st) == 0; }
inline bool is_directory(const path& p) { struct stat st; return ::stat(p.c_str(), &st) == 0 && S_ISDIR(st.st_mode); }
inline bool create_directory(const path& p) { return ::mkdir(p.c_str(), 0755) == 0; }
inline bool create_directories(const path& p) {
  std::string s = p.string(), cur; bool made = false;
  for (std::string::size_type i = 0; i <= s.size(); ++i) {
    if (i == s.size() || s[i] == '/') { if (!cur.empty() && !exists(path(cur))) made = create_directory(path(cur)) || made; }
    if (i < s.size()) cur += s[i];
  }
  return made;
}
}}
#endif
