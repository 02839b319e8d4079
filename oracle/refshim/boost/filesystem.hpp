// boost/filesystem.hpp -- HOST STAND-IN (TEST INFRASTRUCTURE: the reference-pinned oracle under
// oracle/_ref).  The reference uses boost::filesystem for path joining, exists() and file streams
// opened on a path; Boost is not installed here.  This is that small part of the documented
// interface over std::filesystem.
#ifndef REFSHIM_BOOST_FILESYSTEM_HPP_
#define REFSHIM_BOOST_FILESYSTEM_HPP_

#include <filesystem>
#include <fstream>
#include <ostream>
#include <string>

namespace boost {
namespace filesystem {

class path {
 public:
  path() = default;
  path(const char *s) : p_(s) {}
  path(const std::string &s) : p_(s) {}
  path(const std::filesystem::path &p) : p_(p) {}
  std::string string() const { return p_.string(); }
  path operator/(const path &o) const { return path(p_ / o.p_); }
  const std::filesystem::path &native_path() const { return p_; }

 private:
  std::filesystem::path p_;
};
inline std::ostream &operator<<(std::ostream &os, const path &p) { return os << '"' << p.string() << '"'; }
inline bool exists(const path &p) { return std::filesystem::exists(p.native_path()); }
inline bool create_directories(const path &p) { return std::filesystem::create_directories(p.native_path()); }

class ifstream : public std::ifstream {
 public:
  ifstream() = default;
  explicit ifstream(const path &p, std::ios_base::openmode m = std::ios_base::in) : std::ifstream(p.string(), m) {}
};
class ofstream : public std::ofstream {
 public:
  ofstream() = default;
  explicit ofstream(const path &p, std::ios_base::openmode m = std::ios_base::out) : std::ofstream(p.string(), m) {}
};

}  // namespace filesystem
}  // namespace boost

#endif
