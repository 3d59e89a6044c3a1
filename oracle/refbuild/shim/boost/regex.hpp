// std::regex stand-in for boost::regex.  Boost's default (perl) syntax lets '.'
// match a newline and std::regex's ECMAScript syntax does not, so unescaped '.'
// outside bracket expressions is rewritten to [\s\S]; the boost-only "\m"
// escape is dropped.
#pragma once
#include <regex>
#include <string>
namespace boost {
inline std::string regex_shim_translate(const std::string& in) {
  std::string out; bool in_class = false;
  for (size_t i = 0; i < in.size(); ++i) {
    char c = in[i];
    if (c == '\\' && i + 1 < in.size()) {
      if (in[i + 1] == 'm') { ++i; continue; }
      out += c; out += in[++i]; continue;
    }
    if (in_class) { if (c == ']') in_class = false; out += c; continue; }
    if (c == '[') { in_class = true; out += c; continue; }
    if (c == '.') { out += "[\\s\\S]"; continue; }
    out += c;
  }
  return out;
}
class regex : public std::regex {
public:
  regex() {}
  regex(const char* s) : std::regex(regex_shim_translate(s)) {}
  regex(const std::string& s) : std::regex(regex_shim_translate(s)) {}
};
using std::cmatch;
using std::smatch;
template <class... A> bool regex_search(A&&... a) { return std::regex_search(std::forward<A>(a)...); }
template <class... A> bool regex_match(A&&... a) { return std::regex_match(std::forward<A>(a)...); }
}
