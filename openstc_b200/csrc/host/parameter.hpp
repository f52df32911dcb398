// Typed key/value store for the nine setup files of a case directory.
//
// Mirrors the behaviour of OpenSTC's cfd::Parameter (src/Parameter.h:15-84,
// src/Parameter.cpp:21-168): one "type key = value" entry per line, first
// definition of a key wins, "array <type> name { ... }" and
// "struct name { ... }" blocks, and the derived keys ngg / n_var / n_turb /
// n_scalar computed after all files are read.
#pragma once

#include <map>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <variant>
#include <vector>

namespace ostc {

using StructValue = std::variant<std::string, int, double>;
using StructMap = std::map<std::string, StructValue>;

class ParameterError : public std::runtime_error {
 public:
  using std::runtime_error::runtime_error;
};

class Parameter {
 public:
  Parameter() = default;

  // Reads <case_dir>/input_files/setup/{0,1,2,3,4,5,6,8,9}_*.txt in the
  // reference's order and derives ngg, n_var, n_turb, n_scalar, step.
  explicit Parameter(const std::string &case_dir);

  // Parses one setup file (used by tests and by the surrogate settings file).
  void read_file(const std::string &path);

  int &get_int(const std::string &k);
  int get_int(const std::string &k) const;
  double &get_real(const std::string &k);
  double get_real(const std::string &k) const;
  bool get_bool(const std::string &k) const;
  const std::string &get_string(const std::string &k) const;
  const StructMap &get_struct(const std::string &k) const;
  const std::vector<std::string> &get_string_array(const std::string &k) const;
  const std::vector<double> &get_real_array(const std::string &k) const;
  const std::vector<int> &get_int_array(const std::string &k) const;

  bool has_int(const std::string &k) const { return ints_.count(k) != 0; }
  bool has_real(const std::string &k) const { return reals_.count(k) != 0; }
  bool has_bool(const std::string &k) const { return bools_.count(k) != 0; }
  bool has_string(const std::string &k) const { return strings_.count(k) != 0; }
  bool has_struct(const std::string &k) const { return structs_.count(k) != 0; }

  // update_parameter overloads of the reference: overwrite (not emplace).
  void set(const std::string &k, int v) { ints_[k] = v; }
  void set(const std::string &k, double v) { reals_[k] = v; }
  void set_bool(const std::string &k, bool v) { bools_[k] = v; }
  void set(const std::string &k, const std::vector<double> &v) { real_arrays_[k] = v; }

  const std::string &case_dir() const { return case_dir_; }

 private:
  void derive_keys();

  std::string case_dir_{"."};
  std::unordered_map<std::string, int> ints_;
  std::unordered_map<std::string, double> reals_;
  std::unordered_map<std::string, bool> bools_;
  std::unordered_map<std::string, std::string> strings_;
  std::unordered_map<std::string, std::vector<int>> int_arrays_;
  std::unordered_map<std::string, std::vector<double>> real_arrays_;
  std::unordered_map<std::string, std::vector<std::string>> string_arrays_;
  std::unordered_map<std::string, StructMap> structs_;
};

// Helpers to read struct members with the reference's std::get semantics
// (a member stored with another type is an error, a missing one throws).
double struct_real(const StructMap &s, const std::string &k);
int struct_int(const StructMap &s, const std::string &k);
const std::string &struct_string(const StructMap &s, const std::string &k);

}  // namespace ostc
