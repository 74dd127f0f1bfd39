// gs_util.h -- string conventions of the script front end.
//
// The reference passes every parameter as a string and converts with a small
// set of operators (include/datamain.th:36-62): `s >> x` takes the first
// space-separated word of s into x and removes it; `s >>= x` reads the first
// word without consuming it; `s <<= v` overwrites s with v printed by a
// default ostream (six significant digits).  The front end keeps those
// meanings because scripts and info lines depend on them.
#pragma once
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>

namespace gsfe {

// first word of s (leading spaces skipped); s keeps the rest
inline std::string take_word(std::string& s) {
  size_t b = s.find_first_not_of(' ');
  if (b == std::string::npos) {
    s.clear();
    return "";
  }
  s.erase(0, b);
  size_t e = s.find(' ');
  std::string w;
  if (e == std::string::npos) {
    w = s;
    s.clear();
  } else {
    w = s.substr(0, e);
    s.erase(0, e + 1);
  }
  return w;
}

// s >> x: parse the first word into x (x unchanged if the word does not parse)
template <class T> std::string& operator>>(std::string& s, T& x) {
  std::string w = take_word(s);
  std::istringstream is(w);
  T v;
  if (is >> v) x = v;
  return s;
}
inline std::string& operator>>(std::string& s, std::string& x) {
  x = take_word(s);
  return s;
}

// s >>= x: read the first word without consuming s; returns the rest
template <class T> std::string operator>>=(std::string s, T& x) {
  s >> x;
  return s;
}

template <class T> std::string to_string6(const T& v) {
  std::ostringstream os;
  os << v;
  return os.str();
}

// s <<= v
template <class T> std::string& operator<<=(std::string& s, const T& v) {
  s = to_string6(v);
  return s;
}

inline double to_real(const std::string& s) {
  std::string t = s;
  double x = 0;
  t >> x;
  return x;
}

// stdout + <script>.log (src/log_error.h:11-30); `on` only controls the echo
// of script lines, messages are always written
class Log {
 public:
  bool on = true;
  std::ofstream file;
  void open(const std::string& script) { file.open(script + ".log"); }
  template <class T> Log& operator<<(const T& v) {
    std::cout << v;
    if (file) file << v;
    return *this;
  }
  void flush() {
    std::cout.flush();
    if (file) file.flush();
  }
};

Log& log();

// return codes of the script engine (src/pub.h:17-22)
constexpr int kNormal = 0, kErr = -1, kBreak = -2, kQuit = -3, kUnknown = -4, kIncomplete = -5;

}  // namespace gsfe
