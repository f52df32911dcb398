#include "parameter.hpp"

#include <fstream>
#include <sstream>

#include "text.hpp"

namespace ostc {

namespace {
// Setup files in the order the reference reads them (src/Parameter.h:64-74).
const char *kSetupFiles[9] = {
    "0_global_control.txt",   "1_grid_information.txt", "2_scheme.txt",
    "3_species_reactions.txt", "4_laminar_turbulent.txt", "5_boundary_condition.txt",
    "6_post_process.txt",     "8_initialization.txt",   "9_transport_property.txt"};

// Reads whitespace tokens of one line into arr until "}" (returns false: the
// array is complete) or "//" / end of line (returns true: continue on the next
// line).  src/Parameter.cpp:119-142.
template <typename T>
bool collect_tokens(std::istringstream &line, std::vector<T> &arr) {
  std::string tok;
  while (line >> tok) {
    if (tok == "}") return false;
    if (tok == "//") return true;
    if constexpr (std::is_same_v<T, double>) {
      arr.push_back(std::stod(tok));
    } else if constexpr (std::is_same_v<T, int>) {
      arr.push_back(std::stoi(tok));
    } else {
      arr.push_back(tok);
    }
  }
  return true;
}

template <typename T>
void read_array_body(std::ifstream &file, std::istringstream &line, std::vector<T> &arr) {
  std::string input;
  while (collect_tokens(line, arr)) {
    if (!getline_trimmed(file, input, line)) break;
  }
}
}  // namespace

Parameter::Parameter(const std::string &case_dir) : case_dir_(case_dir) {
  for (const char *name : kSetupFiles) {
    read_file(case_dir_ + "/input_files/setup/" + name);
  }
  derive_keys();
}

void Parameter::read_file(const std::string &path) {
  std::ifstream file(path);
  if (!file) throw ParameterError("cannot open setup file " + path);
  std::string input, type, key, eq;
  std::istringstream line;
  while (std::getline(file, input)) {
    // Comment and blank lines are recognised only at column 0, as in
    // src/Parameter.cpp:61-63 (no trimming).
    if (input.empty() || input.rfind("//", 0) == 0 || input.rfind("!", 0) == 0) continue;
    line.clear();
    line.str(input);
    type.clear();
    key.clear();
    eq.clear();
    line >> type >> key >> eq;
    if (type == "int") {
      int v{};
      line >> v;
      ints_.emplace(key, v);
    } else if (type == "real") {
      double v{};
      line >> v;
      reals_.emplace(key, v);
    } else if (type == "bool") {
      bool v{};
      line >> v;
      bools_.emplace(key, v);
    } else if (type == "string") {
      std::string v;
      line >> v;
      strings_.emplace(key, v);
    } else if (type == "array") {
      // "array <elem-type> <name> {": eq holds the name here.
      const std::string name = eq;
      std::string brace;
      if (key == "int") {
        std::vector<int> arr;
        line >> brace;
        read_array_body(file, line, arr);
        int_arrays_.emplace(name, arr);
      } else if (key == "real") {
        std::vector<double> arr;
        line >> brace;
        read_array_body(file, line, arr);
        real_arrays_.emplace(name, arr);
      } else if (key == "string") {
        std::vector<std::string> arr;
        // The reference consumes two tokens here (src/Parameter.cpp:100);
        // a first value written on the "{" line is therefore dropped.
        line >> brace >> brace;
        read_array_body(file, line, arr);
        string_arrays_.emplace(name, arr);
      }
    } else if (type == "struct") {
      StructMap members;
      std::string row, mtype, mname, meq;
      std::istringstream ls;
      while (getline_trimmed(file, row, ls)) {
        mtype.clear();
        ls >> mtype;
        if (mtype == "}") break;  // the closing brace must stand on its own line
        mname.clear();
        meq.clear();
        if (mtype == "string") {
          std::string v;
          ls >> mname >> meq >> v;
          members.emplace(mname, v);
        } else if (mtype == "int") {
          int v{};
          ls >> mname >> meq >> v;
          members.emplace(mname, v);
        } else if (mtype == "real") {
          double v{};
          ls >> mname >> meq >> v;
          members.emplace(mname, v);
        }
      }
      structs_.emplace(key, members);
    }
  }
}

void Parameter::derive_keys() {
  // src/Parameter.cpp:21-55.
  ints_.emplace("step", 0);
  ints_.emplace("ngg", 2);
  if (get_int("inviscid_scheme") / 10 == 5) set("ngg", 3);
  set("n_var", 5);
  set("n_turb", 0);
  int n_scalar = 0;
  if (bools_["turbulence"]) {
    if (ints_["turbulence_method"] == 1) {
      if (ints_["RANS_model"] == 1) {
        set("n_turb", 1);
        set("n_var", 6);
        n_scalar += 1;
      } else {
        set("n_turb", 2);
        set("n_var", 7);
        n_scalar += 2;
      }
    }
  } else {
    set("RANS_model", 0);
  }
  set("n_scalar", n_scalar);
  ints_.emplace("myid", 0);
  ints_.emplace("n_proc", 1);
}

#define OSTC_GET(map, kind)                                                           \
  auto it = map.find(k);                                                              \
  if (it == map.end()) throw ParameterError(std::string("missing ") + kind + " key '" + k + "'"); \
  return it->second;

int &Parameter::get_int(const std::string &k) { OSTC_GET(ints_, "int") }
int Parameter::get_int(const std::string &k) const { OSTC_GET(ints_, "int") }
double &Parameter::get_real(const std::string &k) { OSTC_GET(reals_, "real") }
double Parameter::get_real(const std::string &k) const { OSTC_GET(reals_, "real") }
bool Parameter::get_bool(const std::string &k) const { OSTC_GET(bools_, "bool") }
const std::string &Parameter::get_string(const std::string &k) const { OSTC_GET(strings_, "string") }
const StructMap &Parameter::get_struct(const std::string &k) const { OSTC_GET(structs_, "struct") }
const std::vector<std::string> &Parameter::get_string_array(const std::string &k) const {
  OSTC_GET(string_arrays_, "string array")
}
const std::vector<double> &Parameter::get_real_array(const std::string &k) const {
  OSTC_GET(real_arrays_, "real array")
}
const std::vector<int> &Parameter::get_int_array(const std::string &k) const {
  OSTC_GET(int_arrays_, "int array")
}
#undef OSTC_GET

double struct_real(const StructMap &s, const std::string &k) {
  auto it = s.find(k);
  if (it == s.end()) throw ParameterError("struct member '" + k + "' missing");
  if (!std::holds_alternative<double>(it->second))
    throw ParameterError("struct member '" + k + "' is not a real");
  return std::get<double>(it->second);
}
int struct_int(const StructMap &s, const std::string &k) {
  auto it = s.find(k);
  if (it == s.end()) throw ParameterError("struct member '" + k + "' missing");
  if (!std::holds_alternative<int>(it->second))
    throw ParameterError("struct member '" + k + "' is not an int");
  return std::get<int>(it->second);
}
const std::string &struct_string(const StructMap &s, const std::string &k) {
  auto it = s.find(k);
  if (it == s.end()) throw ParameterError("struct member '" + k + "' missing");
  if (!std::holds_alternative<std::string>(it->second))
    throw ParameterError("struct member '" + k + "' is not a string");
  return std::get<std::string>(it->second);
}

}  // namespace ostc
