// CHEMKIN-format species / thermodynamic / transport / reaction reader.
//
// Behaviour follows OpenSTC's cfd::Species and cfd::Reaction
// (src/ChemData.h:8-69, src/ChemData.cpp:11-614) including its quirks:
//   * the global "T_low T_mid T_high" line of therm.dat does not change the
//     per-species defaults (300/1000/5000), only the species' own line does;
//   * the main-line activation energy is divided by R_c, the LOW and REV ones
//     are not (src/ChemData.cpp:486-487 vs :588-592);
//   * DUPLICATE pairs merge into one reaction of type 3 whose second Arrhenius
//     set goes to (A2, b2, Ea2) (src/ChemData.cpp:389-424);
//   * stoichiometric coefficients are a single leading digit.
#pragma once

#include <map>
#include <string>
#include <vector>

#include "parameter.hpp"

namespace ostc {

constexpr double kRu = 8314.462618;       // J/(kmol K)      src/Constants.h:18
constexpr double kRc = 1.98720425864083;  // cal/(mol K)     src/Constants.h:20
constexpr double kGammaAir = 1.4;         //                 src/Constants.h:22
constexpr double kPatm = 101325.0;        // Pa              src/Constants.h:24
constexpr double kMwAir = 28.9647;        // kg/kmol         src/Constants.h:27

// Standard atomic weight of an element symbol (upper case), -1 if unknown.
double atomic_weight(const std::string &symbol);

struct Species {
  Species() = default;
  explicit Species(Parameter &parameter);

  int n_spec = 0;
  std::map<std::string, int> spec_list;  // name -> index (file order)
  std::map<std::string, int> elem_list;  // element -> column (file order)
  std::vector<int> elem_comp;            // [n_spec][n_elem]
  std::vector<double> mw;                // kg/kmol
  std::vector<double> t_low, t_mid, t_high;
  std::vector<double> low_coeff, high_coeff;  // [n_spec][7]
  std::vector<double> lj_potent_inv, vis_coeff;
  std::vector<double> wj_div_wi_quarter;      // (W_j/W_i)^0.25           [n][n]
  std::vector<double> sqrt_wi_div_wj_8;       // 1/sqrt(8(1+W_i/W_j))     [n][n]

  int n_elem() const { return static_cast<int>(elem_list.size()); }
  // cp of every species at temperature t (J/(kg K)), src/ChemData.cpp:100-118.
  void compute_cp(double t, double *cp) const;
  // Mixture viscosity by Wilke's rule, host variant of src/Transport.cu:11-38.
  double mixture_viscosity(double t, double mw_total, const double *Y) const;

 private:
  void resize(int ns, int ne);
  bool read_therm(std::ifstream &f, bool inside_mechanism);
  void read_tran(std::ifstream &f);
};

struct Reaction {
  Reaction() = default;
  Reaction(Parameter &parameter, const Species &species);

  int n_reac = 0;
  int n_spec = 0;
  // 0 irreversible, 1 reversible, 2 REV, 3 DUP, 4 third body, 5 Lindemann,
  // 6 Troe (3 parameters), 7 Troe (4 parameters).  src/ChemData.h:48-56
  std::vector<int> label;
  std::vector<int> stoi_f, stoi_b;  // [n_reac][n_spec]
  std::vector<int> order;           // sum(products) - sum(reactants)
  std::vector<double> A, b, Ea, A2, b2, Ea2;
  std::vector<double> third_body;   // [n_reac][n_spec], default 1
  std::vector<double> troe_alpha, troe_t3, troe_t1, troe_t2;

 private:
  void resize(int nr, int ns);
  void parse_equation(std::string input, int idx, const Species &sp);
  std::string read_auxiliary(std::ifstream &f, int idx, const Species &sp, bool &is_dup);
};

}  // namespace ostc
