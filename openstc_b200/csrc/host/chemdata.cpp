#include "chemdata.hpp"

#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>

#include "text.hpp"

namespace ostc {

double atomic_weight(const std::string &symbol) {
  // IUPAC abridged standard atomic weights; the subset a combustion or
  // air-chemistry mechanism can name.  Values are the ones the reference
  // tabulates (src/Element.cpp:13-166) so that W_k agrees to the last bit.
  static const std::map<std::string, double> table = {
      {"H", 1.008},        {"HE", 4.002602},     {"LI", 6.94},        {"BE", 9.0121831},
      {"B", 10.81},        {"C", 12.011},        {"N", 14.007},       {"O", 15.999},
      {"F", 18.998403163}, {"NE", 20.1797},      {"NA", 22.98976928}, {"MG", 24.305},
      {"AL", 26.9815384},  {"SI", 28.085},       {"P", 30.973761998}, {"S", 32.06},
      {"CL", 35.45},       {"AR", 39.95},        {"K", 39.0983},      {"CA", 40.078},
      {"TI", 47.867},      {"CR", 51.9961},      {"FE", 55.845},      {"NI", 58.6934},
      {"CU", 63.546},      {"KR", 83.798},       {"XE", 131.293},
      // isotopes and the electron (src/Element.cpp:129-133)
      {"D", 2.0141017781}, {"E", 9.1093837015e-31 * 6.02214076e26}};
  auto it = table.find(symbol);
  return it == table.end() ? -1.0 : it->second;
}

// ----------------------------------------------------------------- Species
void Species::resize(int ns, int ne) {
  n_spec = ns;
  elem_comp.assign(static_cast<size_t>(ns) * ne, 0);
  mw.assign(ns, 0.0);
  t_low.assign(ns, 300.0);
  t_mid.assign(ns, 1000.0);
  t_high.assign(ns, 5000.0);
  low_coeff.assign(static_cast<size_t>(ns) * 7, 0.0);
  high_coeff.assign(static_cast<size_t>(ns) * 7, 0.0);
  lj_potent_inv.assign(ns, 0.0);
  vis_coeff.assign(ns, 0.0);
  wj_div_wi_quarter.assign(static_cast<size_t>(ns) * ns, 0.0);
  sqrt_wi_div_wj_8.assign(static_cast<size_t>(ns) * ns, 0.0);
}

Species::Species(Parameter &parameter) {
  parameter.set("n_spec", 0);
  if (!parameter.get_bool("species")) return;
  const std::string root = parameter.case_dir() + "/input_files/";
  const std::string mech = root + parameter.get_string("mechanism_file");
  std::ifstream file(mech);
  if (!file) throw ParameterError("cannot open mechanism file " + mech);
  std::string tok;
  auto skip_comment = [&](const std::string &t) {
    if (!t.empty() && t[0] == '!') {
      std::getline(file, tok);
      return true;
    }
    return false;
  };
  while (file >> tok) {
    if (skip_comment(tok)) continue;
    if (tok == "ELEMENTS" || tok == "ELEM") break;
  }
  int ne = 0;
  while (file >> tok) {
    if (skip_comment(tok)) continue;
    tok = upper(tok);
    if (tok == "END") continue;
    if (tok == "SPECIES" || tok == "SPEC") break;
    elem_list.emplace(tok, ne++);
  }
  int ns = 0;
  bool therm_inside = false;
  while (file >> tok) {
    if (skip_comment(tok)) continue;
    tok = upper(tok);
    if (tok == "END") continue;
    if (tok == "REACTIONS" || tok == "REAC") break;
    if (tok == "THERMO") {
      therm_inside = true;
      break;
    }
    spec_list.emplace(tok, ns++);
  }
  resize(ns, ne);
  if (ns > 20)
    throw ParameterError("mechanism has " + std::to_string(ns) +
                         " species; at most 20 are supported (MAX_SPEC_NUMBER)");
  parameter.set("n_spec", ns);
  parameter.set("n_var", parameter.get_int("n_var") + ns);
  parameter.set("n_scalar", parameter.get_int("n_scalar") + ns);

  if (!therm_inside) {
    file.close();
    const std::string th = root + parameter.get_string("therm_file");
    file.open(th);
    if (!file) throw ParameterError("cannot open thermo file " + th);
  }
  const bool tran_inside = read_therm(file, therm_inside);
  if (!tran_inside) {
    file.close();
    const std::string tr = root + parameter.get_string("transport_file");
    file.open(tr);
    if (!file) throw ParameterError("cannot open transport file " + tr);
  }
  read_tran(file);
}

bool Species::read_therm(std::ifstream &f, bool inside_mechanism) {
  std::string input;
  if (!inside_mechanism) read_until(f, input, {"THERMO"}, Fold::upper);
  // The global temperature line: read and discarded, exactly as the
  // reference's resize() on already-sized vectors leaves the defaults.
  while (std::getline(f, input)) {
    if (input.empty() || input[0] == '!') continue;
    break;
  }
  std::vector<int> done;
  int n_read = 0;
  bool tran_inside = false;
  std::istringstream line;
  std::string key;
  while (getline_trimmed(f, input, line, Fold::upper)) {
    if (input.empty() || input[0] == '!') continue;
    key.clear();
    line >> key;
    if (key == "END") continue;
    if (key == "REACTIONS" || input == "REAC") break;
    if (key == "TRANSPORT" || key == "TRAN") {
      tran_inside = true;
      break;
    }
    if (n_read >= n_spec) continue;
    {
      std::istringstream nm(input.substr(0, std::min<size_t>(18, input.size())));
      key.clear();
      nm >> key;
    }
    auto it = spec_list.find(key);
    if (it == spec_list.end()) {
      for (int r = 0; r < 3; ++r) getline_trimmed(f, input);
      continue;
    }
    const int sp = it->second;
    if (std::find(done.begin(), done.end(), sp) != done.end()) {
      for (int r = 0; r < 3; ++r) getline_trimmed(f, input);
      getline_trimmed(f, input, line, Fold::upper);  // the reference consumes one more line here
      continue;
    }
    auto field = [&](size_t pos, size_t len) { return input.size() > pos ? input.substr(pos, len) : std::string(); };
    t_low[sp] = std::stod(field(45, 10));
    t_high[sp] = std::stod(field(55, 10));
    {
      std::istringstream tm(field(65, 10));
      std::string v;
      if (tm >> v) t_mid[sp] = std::stod(v);
    }
    for (int e = 0; e < 4; ++e) {
      std::string comp = field(24 + 5 * e, 5);
      trim_left(comp);
      if (comp.empty() || comp[0] == '0') break;
      std::istringstream cs(comp);
      std::string el;
      int cnt = 0;
      cs >> el >> cnt;
      auto eit = elem_list.find(el);
      if (eit == elem_list.end()) eit = elem_list.emplace(el, 0).first;  // reference: operator[]
      elem_comp[static_cast<size_t>(sp) * n_elem() + eit->second] = cnt;
    }
    double w = 0.0;
    for (const auto &[el, col] : elem_list) {
      w += atomic_weight(el) * elem_comp[static_cast<size_t>(sp) * n_elem() + col];
    }
    mw[sp] = w;
    // Three lines of five 15-character fields (raw lines, not trimmed).
    double c[15];
    for (int r = 0; r < 3; ++r) {
      std::getline(f, input);
      const int nf = (r == 2) ? 4 : 5;
      for (int q = 0; q < nf; ++q) c[r * 5 + q] = std::stod(input.substr(15 * q, 15));
    }
    double *hi = &high_coeff[static_cast<size_t>(sp) * 7];
    double *lo = &low_coeff[static_cast<size_t>(sp) * 7];
    for (int q = 0; q < 5; ++q) hi[q] = c[q];
    hi[5] = c[5];
    hi[6] = c[6];
    lo[0] = c[7];
    lo[1] = c[8];
    lo[2] = c[9];
    lo[3] = c[10];
    lo[4] = c[11];
    lo[5] = c[12];
    lo[6] = c[13];
    done.push_back(sp);
    ++n_read;
  }
  if (n_read < n_spec)
    std::fprintf(stderr, "thermodynamic data for %d of %d species only\n", n_read, n_spec);
  return tran_inside;
}

void Species::read_tran(std::ifstream &f) {
  std::string input, key;
  std::istringstream line;
  std::vector<int> done;
  int n_read = 0;
  while (getline_trimmed(f, input, line, Fold::upper)) {
    if (input.empty() || input[0] == '!') continue;
    key.clear();
    line >> key;
    if (key.rfind("END", 0) == 0 || key.rfind("REACTIONS", 0) == 0 || key.rfind("REAC", 0) == 0) break;
    auto it = spec_list.find(key);
    if (it == spec_list.end()) continue;
    if (n_read >= n_spec) break;
    const int sp = it->second;
    if (std::find(done.begin(), done.end(), sp) != done.end()) continue;
    std::istringstream ls(input);
    double geometry = 0, eps_k = 0, sigma = 0;
    ls >> key >> geometry >> eps_k >> sigma;
    lj_potent_inv[sp] = 1.0 / eps_k;
    vis_coeff[sp] = 2.6693e-6 * std::sqrt(mw[sp]) / (sigma * sigma);
    done.push_back(sp);
    ++n_read;
  }
  if (n_read < n_spec) std::fprintf(stderr, "transport data for %d of %d species only\n", n_read, n_spec);
  for (int i = 0; i < n_spec; ++i) {
    for (int j = 0; j < n_spec; ++j) {
      wj_div_wi_quarter[i * n_spec + j] = std::pow(mw[j] / mw[i], 0.25);
      sqrt_wi_div_wj_8[i * n_spec + j] = 1.0 / std::sqrt(8 * (1 + mw[i] / mw[j]));
    }
  }
}

void Species::compute_cp(double t, double *cp) const {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t;
  for (int i = 0; i < n_spec; ++i) {
    if (t < t_low[i]) {
      const double tt = t_low[i], tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt;
      const double *c = &low_coeff[i * 7];
      cp[i] = c[0] + c[1] * tt + c[2] * tt2 + c[3] * tt3 + c[4] * tt4;
    } else {
      const double *c = (t < t_mid[i]) ? &low_coeff[i * 7] : &high_coeff[i * 7];
      cp[i] = c[0] + c[1] * t + c[2] * t2 + c[3] * t3 + c[4] * t4;
    }
    cp[i] *= kRu / mw[i];
  }
}

double Species::mixture_viscosity(double t, double mw_total, const double *Y) const {
  std::vector<double> x(n_spec), mu(n_spec), phi(static_cast<size_t>(n_spec) * n_spec);
  for (int i = 0; i < n_spec; ++i) {
    x[i] = Y[i] * mw_total / mw[i];
    const double tdl = t * lj_potent_inv[i];
    const double omega = 1.147 * std::pow(tdl, -0.145) + std::pow(tdl + 0.5, -2);
    mu[i] = vis_coeff[i] * std::sqrt(t) / omega;
  }
  for (int i = 0; i < n_spec; ++i) {
    for (int j = 0; j < n_spec; ++j) {
      if (i == j) {
        phi[i * n_spec + j] = 1.0;
      } else {
        const double num = 1 + std::sqrt(mu[i] / mu[j]) * wj_div_wi_quarter[i * n_spec + j];
        phi[i * n_spec + j] = num * num * sqrt_wi_div_wj_8[i * n_spec + j];
      }
    }
  }
  double visc = 0;
  for (int i = 0; i < n_spec; ++i) {
    double den = 0;
    for (int j = 0; j < n_spec; ++j) den += phi[i * n_spec + j] * x[j];
    visc += mu[i] * x[i] / den;
  }
  return visc;
}

// ---------------------------------------------------------------- Reaction
void Reaction::resize(int nr, int ns) {
  n_reac = nr;
  n_spec = ns;
  label.resize(nr, 1);
  stoi_f.resize(static_cast<size_t>(nr) * ns, 0);
  stoi_b.resize(static_cast<size_t>(nr) * ns, 0);
  order.resize(nr, 0);
  A.resize(nr, 0);
  b.resize(nr, 0);
  Ea.resize(nr, 0);
  A2.resize(nr, 0);
  b2.resize(nr, 0);
  Ea2.resize(nr, 0);
  third_body.resize(static_cast<size_t>(nr) * ns, 1.0);
  troe_alpha.resize(nr, 0);
  troe_t3.resize(nr, 0);
  troe_t1.resize(nr, 0);
  troe_t2.resize(nr, 0);
}

Reaction::Reaction(Parameter &parameter, const Species &sp) {
  parameter.set("n_reac", 0);
  n_spec = sp.n_spec;
  if (!parameter.get_bool("species") || !parameter.get_bool("reaction")) return;
  const std::string mech = parameter.case_dir() + "/input_files/" + parameter.get_string("mechanism_file");
  std::ifstream file(mech);
  if (!file) throw ParameterError("cannot open mechanism file " + mech);
  std::string input;
  read_until(file, input, {"REACTIONS", "REAC"}, Fold::keep);
  const int ns = sp.n_spec;
  resize(100, ns);
  int has_read = 0;
  std::vector<int> dup_open;
  std::istringstream line;
  getline_trimmed(file, input, line, Fold::upper);
  int guard = 0;
  while (input != "END") {
    if (input.empty() || input[0] == '!') {
      // The reference loops forever on a blank line here; read on instead.
      if (!getline_trimmed(file, input, line, Fold::upper) || ++guard > 100000) break;
      continue;
    }
    if (has_read >= n_reac) resize(n_reac + 100, ns);
    parse_equation(input, has_read, sp);
    bool is_dup = false;
    input = read_auxiliary(file, has_read, sp, is_dup);
    if (is_dup) {
      int found = -1;
      for (size_t r = 0; r < dup_open.size(); ++r) {
        const int d = dup_open[r];
        bool same = true;
        for (int i = 0; i < ns; ++i) {
          if (stoi_f[d * ns + i] != stoi_f[has_read * ns + i] || stoi_b[d * ns + i] != stoi_b[has_read * ns + i]) {
            same = false;
            break;
          }
        }
        if (same) {
          found = static_cast<int>(r);
          break;
        }
      }
      if (found >= 0) {
        const int d = dup_open[found];
        A2[d] = A[has_read];
        b2[d] = b[has_read];
        Ea2[d] = Ea[has_read];
        dup_open.erase(dup_open.begin() + found);
        for (int i = 0; i < ns; ++i) {
          stoi_f[has_read * ns + i] = 0;
          stoi_b[has_read * ns + i] = 0;
        }
        label[has_read] = 1;
        order[has_read] = 0;
      } else {
        dup_open.push_back(has_read);
        ++has_read;
      }
      continue;
    }
    ++has_read;
  }
  // Shrink to the reactions read; rows are contiguous so the leading part stays.
  label.resize(has_read);
  stoi_f.resize(static_cast<size_t>(has_read) * ns);
  stoi_b.resize(static_cast<size_t>(has_read) * ns);
  order.resize(has_read);
  for (auto *v : {&A, &b, &Ea, &A2, &b2, &Ea2, &troe_alpha, &troe_t3, &troe_t1, &troe_t2}) v->resize(has_read);
  third_body.resize(static_cast<size_t>(has_read) * ns);
  n_reac = has_read;
  parameter.set("n_reac", n_reac);
}

void Reaction::parse_equation(std::string input, int idx, const Species &sp) {
  const auto lp = input.find("(+");
  const auto cat = input.find("+M");
  if (cat != std::string::npos) {
    label[idx] = 4;
    if (lp != std::string::npos) {
      label[idx] = 5;
      const auto rp = input.find(')', lp);
      input.erase(lp, rp + 1 - lp);
      const auto lp2 = input.find("(+");
      const auto rp2 = input.find_last_of(')');
      input.erase(lp2, rp2 + 1 - lp2);
    } else {
      input.erase(cat, 2);
      input.erase(input.find("+M"), 2);
    }
  }
  auto small = input.find('<');
  const auto eq = input.find('=');
  if (small == std::string::npos) small = eq;
  if (small != std::string::npos) std::replace(input.begin(), input.begin() + small + 1, ' ', '<');
  std::string eqn;
  std::istringstream ls(input);
  ls >> eqn >> A[idx] >> b[idx] >> Ea[idx];
  Ea[idx] /= kRc;

  auto s = eqn.find('<');
  const auto e = eqn.find('=');
  auto g = eqn.find('>');
  if (s == std::string::npos) {
    if (g != std::string::npos) {
      label[idx] = 0;
    } else {
      g = e;
    }
    s = e;
  }
  std::string lhs = eqn.substr(0, s);
  std::string rhs = eqn.substr(g + 1);
  const int ns = sp.n_spec;
  auto spec_index = [&](const std::string &name) {
    auto it = sp.spec_list.find(name);
    if (it == sp.spec_list.end()) throw ParameterError("unknown species '" + name + "' in reaction " + eqn);
    return it->second;
  };
  auto take = [&](std::string &side, bool reactant) {
    for (auto p = side.find('+'); p != std::string::npos; p = side.find('+')) {
      if (reactant && p + 1 < side.size() && side[p + 1] == '+') ++p;
      int nu = 1;
      std::string name;
      if (std::isdigit(static_cast<unsigned char>(side[0]))) {
        nu = side[0] - '0';
        side.erase(0, 1);
        name = side.substr(0, p - 1);
      } else {
        name = side.substr(0, p);
      }
      (reactant ? stoi_f : stoi_b)[static_cast<size_t>(idx) * ns + spec_index(name)] += nu;
      order[idx] += reactant ? -nu : nu;
      side.erase(0, name.size() + 1);
    }
    int nu = 1;
    if (!side.empty() && std::isdigit(static_cast<unsigned char>(side[0]))) {
      nu = side[0] - '0';
      side.erase(0, 1);
    }
    (reactant ? stoi_f : stoi_b)[static_cast<size_t>(idx) * ns + spec_index(side)] += nu;
    order[idx] += reactant ? -nu : nu;
  };
  take(lhs, true);
  take(rhs, false);
}

std::string Reaction::read_auxiliary(std::ifstream &f, int idx, const Species &sp, bool &is_dup) {
  std::string input, key;
  const int ns = sp.n_spec;
  while (getline_trimmed(f, input, Fold::upper)) {
    std::replace(input.begin(), input.end(), '/', ' ');
    std::istringstream ls(input);
    key.clear();
    ls >> key;
    if (input.empty() || input[0] == '!') continue;
    if (key == "END") break;
    if (input.find('=') != std::string::npos) break;
    if (key == "PLOG") continue;
    if (key == "DUPLICATE" || key == "DUP") {
      is_dup = true;
      label[idx] = 3;
      continue;
    }
    if (key == "REV") {
      ls >> A2[idx] >> b2[idx] >> Ea2[idx];
      label[idx] = 2;
    } else if (key == "LOW") {
      ls >> A2[idx] >> b2[idx] >> Ea2[idx];
    } else if (key == "TROE") {
      label[idx] = 6;
      ls >> troe_alpha[idx] >> troe_t3[idx] >> troe_t1[idx];
      std::string t2;
      if (ls >> t2) {
        troe_t2[idx] = std::stod(t2);
        label[idx] = 7;
      }
    } else {
      std::istringstream tb(input);
      std::string name;
      while (tb >> name) {
        double eff = 0;
        tb >> eff;
        auto it = sp.spec_list.find(name);
        if (it == sp.spec_list.end()) throw ParameterError("unknown third-body species '" + name + "'");
        third_body[static_cast<size_t>(idx) * ns + it->second] = eff;
      }
    }
  }
  return input;
}

}  // namespace ostc
