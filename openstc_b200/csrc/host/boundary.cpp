#include "boundary.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>

namespace ostc {

namespace {
double sutherland(double t) { return 1.716e-5 * std::pow(t / 273, 1.5) * (273 + 111) / (t + 111); }

bool has(const StructMap &s, const std::string &k) { return s.find(k) != s.end(); }
}  // namespace

Inflow::Inflow(const std::string &name, const Species &spec, Parameter &parameter) {
  const StructMap &info = parameter.get_struct(name);
  label = struct_int(info, "label");
  if (has(info, "mach")) mach = struct_real(info, "mach");
  if (has(info, "pressure")) pressure = struct_real(info, "pressure");
  if (has(info, "temperature")) temperature = struct_real(info, "temperature");
  if (has(info, "velocity")) velocity = struct_real(info, "velocity");
  if (has(info, "density")) density = struct_real(info, "density");
  if (has(info, "u")) u = struct_real(info, "u");
  if (has(info, "v")) v = struct_real(info, "v");
  if (has(info, "w")) w = struct_real(info, "w");
  const int n_scalar = parameter.get_int("n_scalar");
  sv.assign(n_scalar, 0.0);
  const int ns = spec.n_spec;
  if (ns > 0) {
    for (const auto &[sname, idx] : spec.spec_list)
      if (has(info, sname)) sv[idx] = struct_real(info, sname);
    mw = 0;
    for (int i = 0; i < ns; ++i) mw += sv[i] / spec.mw[i];
    mw = 1 / mw;
  }
  if (temperature < 0) temperature = pressure * mw / (density * kRu);
  viscosity = ns > 0 ? spec.mixture_viscosity(temperature, mw, sv.data()) : sutherland(temperature);
  double gamma = kGammaAir;
  if (ns > 0) {
    std::vector<double> cpi(ns);
    spec.compute_cp(temperature, cpi.data());
    double cp = 0, cv = 0;
    for (int i = 0; i < ns; ++i) {
      cp += sv[i] * cpi[i];
      cv += sv[i] * (cpi[i] - kRu / spec.mw[i]);
    }
    gamma = cp / cv;
  }
  const double c = std::sqrt(gamma * kRu / mw * temperature);
  if (mach < 0) {
    mach = velocity / c;
  } else {
    velocity = mach * c;
  }
  u *= velocity;
  v *= velocity;
  w *= velocity;
  if (density < 0) density = pressure * mw / (kRu * temperature);
  if (parameter.get_int("turbulence_method") == 1 && parameter.get_int("RANS_model") == 2) {
    mut = struct_real(info, "turb_viscosity_ratio") * viscosity;
    if (has(info, "turbulence_intensity")) {
      const double ti = struct_real(info, "turbulence_intensity");
      sv[ns] = 1.5 * velocity * velocity * ti * ti;
      sv[ns + 1] = density * sv[ns] / mut;
    }
  }
  if (name == "freestream") {  // src/BoundCond.cpp:96-105 keys the name literally
    parameter.set("rho_inf", density);
    parameter.set("v_inf", velocity);
    parameter.set("p_inf", pressure);
    parameter.set("sv_inf", sv);
  }
}

void BcRegistry::build(Mesh &mesh, const Species &spec, Parameter &parameter) {
  std::vector<int> labels;
  for (const auto &b : mesh.block)
    for (const auto &f : b.boundary)
      if (std::find(labels.begin(), labels.end(), f.label) == labels.end()) labels.push_back(f.label);
  const std::vector<std::string> empty;
  const auto &names = [&]() -> const std::vector<std::string> & {
    try {
      return parameter.get_string_array("boundary_conditions");
    } catch (const ParameterError &) {
      return empty;
    }
  }();
  for (const auto &bc_name : names) {
    const StructMap &s = parameter.get_struct(bc_name);
    const int lab = struct_int(s, "label");
    auto it = std::find(labels.begin(), labels.end(), lab);
    if (it == labels.end()) continue;
    labels.erase(it);
    const std::string &type = struct_string(s, "type");
    if (type == "wall") wall_labels.push_back(lab);
    else if (type == "inflow") inflow_labels.push_back(lab);
    else if (type == "outflow") outflow_labels.push_back(lab);
    else if (type == "symmetry") symmetry_labels.push_back(lab);
  }
  for (int lab : labels) {
    if (lab == 2) wall_labels.push_back(lab);
    else if (lab == 3) symmetry_labels.push_back(lab);
    else if (lab == 5) inflow_labels.push_back(lab);
    else if (lab == 6) outflow_labels.push_back(lab);
  }
  for (int lab : wall_labels) {
    Wall wl;
    wl.label = lab;
    for (const auto &bc_name : names) {
      const StructMap &s = parameter.get_struct(bc_name);
      if (struct_int(s, "label") != lab) continue;
      if (has(s, "thermal_type")) wl.isothermal = struct_string(s, "thermal_type") == "isothermal";
      if (wl.isothermal) {
        if (has(s, "temperature")) wl.temperature = struct_real(s, "temperature");
        else std::printf("Isothermal wall does not specify wall temperature, is set as 300K in default.\n");
      }
    }
    wall.push_back(wl);
  }
  for (int lab : inflow_labels) {
    bool found = false;
    for (const auto &bc_name : names) {
      const StructMap &s = parameter.get_struct(bc_name);
      if (struct_int(s, "label") != lab) continue;
      inflow.emplace_back(bc_name, spec, parameter);
      found = true;
      break;
    }
    if (!found) throw ParameterError("inflow label " + std::to_string(lab) + " has no struct in boundary_conditions");
  }
  // Application order per block (src/BoundCond.cuh:321-412).
  struct Kind {
    BcType type;
    const std::vector<int> *labels;
  };
  const Kind kinds[4] = {{BcType::outflow, &outflow_labels},
                         {BcType::inflow, &inflow_labels},
                         {BcType::symmetry, &symmetry_labels},
                         {BcType::wall, &wall_labels}};
  for (int b = 0; b < mesh.n_block; ++b) {
    for (const auto &kd : kinds) {
      for (size_t l = 0; l < kd.labels->size(); ++l) {
        for (size_t f = 0; f < mesh[b].boundary.size(); ++f) {
          if (mesh[b].boundary[f].label != (*kd.labels)[l]) continue;
          order.push_back(BcFace{b, static_cast<int>(f), kd.type, static_cast<int>(l)});
        }
      }
    }
  }
  const int ngg = mesh.ngg;
  for (auto &b : mesh.block)
    for (auto &f : b.boundary)
      if (std::find(wall_labels.begin(), wall_labels.end(), f.label) != wall_labels.end())
        for (int q = 0; q < 3; ++q) {
          if (q == f.face) continue;
          f.start[q] += ngg;
          f.end[q] -= ngg;
        }
}

void initialize_from_start(Parameter &parameter, const Mesh &mesh, const Species &spec,
                           std::vector<HostField> &field) {
  const int groups = parameter.get_int("groups_init");
  std::vector<Inflow> inflows;
  inflows.emplace_back(parameter.get_string("default_init"), spec, parameter);
  std::vector<double> xs, xe, ys, ye, zs, ze;
  for (int l = 0; l + 1 < groups; ++l) {
    const std::string nm = "init_cond_" + std::to_string(l);
    const StructMap &p = parameter.get_struct(nm);
    xs.push_back(struct_real(p, "x0"));
    xe.push_back(struct_real(p, "x1"));
    ys.push_back(struct_real(p, "y0"));
    ye.push_back(struct_real(p, "y1"));
    zs.push_back(struct_real(p, "z0"));
    ze.push_back(struct_real(p, "z1"));
    if (has(p, "label")) inflows.emplace_back(struct_string(p, "label"), spec, parameter);
    else inflows.emplace_back(nm, spec, parameter);
  }
  const int n_scalar = parameter.get_int("n_scalar");
  for (int b = 0; b < mesh.n_block; ++b) {
    const Block &B = mesh[b];
    HostField &F = field[b];
    F.e = Extent{B.mx, B.my, B.mz, B.ngg};
    F.n_scalar = n_scalar;
    F.bv.assign(static_cast<size_t>(6 * F.e.size()), 0.0);
    F.sv.assign(static_cast<size_t>(n_scalar * F.e.size()), 0.0);
    const int g = B.ngg;
    for (int i = -g; i < B.mx + g; ++i)
      for (int j = -g; j < B.my + g; ++j)
        for (int k = -g; k < B.mz + g; ++k) {
          size_t pick = 0;
          // The reference tests inflow l against box l (src/Field.cu:41-50)
          // although box l belongs to inflow l+1; boxes past the end never match.
          for (size_t l = 1; l < inflows.size(); ++l) {
            if (l >= xs.size()) break;
            const double x = B.x(i, j, k), y = B.y(i, j, k), z = B.z(i, j, k);
            if (x >= xs[l] && x <= xe[l] && y >= ys[l] && y <= ye[l] && z >= zs[l] && z <= ze[l]) {
              pick = l;
              break;
            }
          }
          const Inflow &in = inflows[pick];
          F.b(i, j, k, 0) = in.density;
          F.b(i, j, k, 1) = in.u;
          F.b(i, j, k, 2) = in.v;
          F.b(i, j, k, 3) = in.w;
          F.b(i, j, k, 4) = in.pressure;
          F.b(i, j, k, 5) = in.temperature;
          for (int l = 0; l < n_scalar; ++l) F.s(i, j, k, l) = in.sv[l];
        }
  }
}

}  // namespace ostc
