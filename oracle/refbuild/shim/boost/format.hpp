// Tiny stand-in for boost::format supporting a single integer argument with a
// printf-style format such as "%05d" (the only form the reference uses).
#pragma once
#include <string>
#include <cstdio>
namespace boost {
class format {
  std::string f_, out_;
public:
  explicit format(const char* f) : f_(f) {}
  format& operator%(int v) { char b[256]; std::snprintf(b, sizeof b, f_.c_str(), v); out_ = b; return *this; }
  std::string str() const { return out_; }
};
inline std::string str(const format& f) { return f.str(); }
}
