// Small text helpers with the semantics the reference's readers rely on
// (src/gxl_lib/MyString.cpp:4-62): left-trimmed lines, optional case folding.
#pragma once

#include <algorithm>
#include <cctype>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace ostc {

inline void trim_left(std::string &s) {
  const auto p = s.find_first_not_of(" \n\t\r\f\v");
  s = (p == std::string::npos) ? std::string() : s.substr(p);
}

inline std::string upper(std::string s) {
  for (auto &c : s) c = static_cast<char>(std::toupper(static_cast<unsigned char>(c)));
  return s;
}

enum class Fold { keep, upper };

// Reads a line, trims its left side, folds case and loads it into `line`.
inline bool getline_trimmed(std::ifstream &f, std::string &input, std::istringstream &line,
                            Fold fold = Fold::keep) {
  if (!std::getline(f, input)) {
    input.clear();
    line.clear();
    line.str(input);
    return false;
  }
  trim_left(input);
  if (fold == Fold::upper) input = upper(input);
  line.clear();
  line.str(input);
  return true;
}

inline bool getline_trimmed(std::ifstream &f, std::string &input, Fold fold = Fold::keep) {
  if (!std::getline(f, input)) {
    input.clear();
    return false;
  }
  trim_left(input);
  if (fold == Fold::upper) input = upper(input);
  return true;
}

// Advances to the first line (trimmed, folded) starting with one of `keys`;
// sets input to "end" when none is found (src/gxl_lib/MyString.cpp:48-75).
inline bool read_until(std::ifstream &f, std::string &input, const std::vector<std::string> &keys,
                       Fold fold = Fold::keep) {
  while (getline_trimmed(f, input, fold)) {
    for (const auto &k : keys)
      if (input.rfind(k, 0) == 0) return true;
  }
  input = "end";
  return false;
}

}  // namespace ostc
