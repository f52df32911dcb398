// Inflow / wall conditions, the boundary-condition registry and the initial
// flow field.
//
// Inflow / Wall follow src/BoundCond.cpp:6-156; the registry follows
// DBoundCond::initialize_bc_on_GPU / link_bc_to_boundaries
// (src/BoundCond.cu:73-250), which fixes the order in which faces are
// applied: every outflow face, then inflow, symmetry and wall faces, each
// type in registration order and each face in (block, face) order.  Wall
// faces lose ngg points at both ends of their tangential ranges.
#pragma once

#include <string>
#include <vector>

#include "chemdata.hpp"
#include "mesh.hpp"

namespace ostc {

struct Inflow {
  Inflow() = default;
  Inflow(const std::string &name, const Species &spec, Parameter &parameter);
  int label = 5;
  double mach = -1, pressure = 101325, temperature = -1, velocity = 0, density = -1;
  double u = 1, v = 0, w = 0;
  double mw = kMwAir, viscosity = 0, mut = 0;
  std::vector<double> sv;  // n_scalar values: Y_k then k, omega
};

struct Wall {
  int label = 2;
  bool isothermal = true;
  double temperature = 300;
};

enum class BcType : int { outflow = 6, inflow = 5, symmetry = 3, wall = 2 };

// One boundary face occurrence in application order.
struct BcFace {
  int block = 0;
  int face_index = 0;  // index into Block::boundary
  BcType type = BcType::outflow;
  int cond = 0;        // index into the inflow or wall list
};

struct BcRegistry {
  std::vector<Inflow> inflow;
  std::vector<Wall> wall;
  std::vector<int> outflow_labels, inflow_labels, symmetry_labels, wall_labels;
  std::vector<BcFace> order;  // application order
  // Builds the registry and trims wall faces of `mesh` in place.
  void build(Mesh &mesh, const Species &spec, Parameter &parameter);
};

// Host copy of one block's primitive state in the reference layout with ngg
// ghost layers: bv = (rho, u, v, w, p, T), sv = (Y_0..Y_ns-1, k, omega).
struct HostField {
  Extent e;
  int n_scalar = 0;
  std::vector<double> bv, sv;
  double &b(int i, int j, int k, int l) { return bv[static_cast<size_t>(l * e.size() + e.at(i, j, k))]; }
  double &s(int i, int j, int k, int l) { return sv[static_cast<size_t>(l * e.size() + e.at(i, j, k))]; }
};

// Fresh start (initial = 0): the default inflow everywhere, patched by the
// init_cond_N boxes (src/Initialize.cu:4-43, src/Field.cu:21-67).  Also sets
// rho_inf / v_inf / p_inf / sv_inf through the "freestream" inflow.
void initialize_from_start(Parameter &parameter, const Mesh &mesh, const Species &spec,
                           std::vector<HostField> &field);

}  // namespace ostc
