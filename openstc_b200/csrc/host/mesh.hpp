// Structured multi-block grid: the "Plot3D with a little variation" reader,
// boundary / inner-face topology, ghost geometry and the central-difference
// Jacobian and metric.
//
// Follows OpenSTC's Mesh / Block / Boundary / InnerFace
// (src/Mesh.h:8-232, src/Mesh.cpp:14-993).  Arrays use the reference's
// column-major layout with negative ghost indices:
//   index(i,j,k) = k*(mx+2g)*(my+2g) + j*(mx+2g) + i + ((mx+2g)*(my+2g) + (mx+2g) + 1)*g
// The metric is stored as nine separate arrays (xi_x, xi_y, xi_z, eta_x, ...,
// zeta_z) instead of the reference's 3x3 struct per point.
#pragma once

#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "parameter.hpp"

namespace ostc {

struct Extent {
  int mx = 1, my = 1, mz = 1, ng = 0;
  int64_t sx() const { return mx + 2 * ng; }
  int64_t sxy() const { return sx() * (my + 2 * ng); }
  int64_t size() const { return sxy() * (mz + 2 * ng); }
  int64_t off() const { return (sxy() + sx() + 1) * ng; }
  int64_t at(int i, int j, int k) const { return k * sxy() + j * sx() + i + off(); }
};

struct Array3 {
  Extent e;
  std::vector<double> v;
  Array3() = default;
  Array3(int mx, int my, int mz, int ng) : e{mx, my, mz, ng}, v(static_cast<size_t>(e.size()), 0.0) {}
  double &operator()(int i, int j, int k) { return v[static_cast<size_t>(e.at(i, j, k))]; }
  double operator()(int i, int j, int k) const { return v[static_cast<size_t>(e.at(i, j, k))]; }
};

// A physical boundary patch (src/Mesh.h:9-33).  Indices are 0-based and the
// tangential ranges include ngg ghost points on each side after registration.
struct Boundary {
  int start[3] = {0, 0, 0};
  int end[3] = {0, 0, 0};
  int label = 0;
  int face = 0;       // 0 i, 1 j, 2 k
  int direction = 1;  // +1: outward normal along +index
  void register_face(int ngg, int dim);
};

// A block-to-block interface on the same process (src/Mesh.h:35-66).
struct InnerFace {
  int start[3], end[3], tstart[3], tend[3];
  int target_block = 0;
  int face = 0, direction = 1, target_face = 0, target_direction = 1;
  int src_tar[3] = {0, 0, 0};
  int loop_dir[3] = {1, 1, 1};
  int target_loop_dir[3] = {1, 1, 1};
  int n_point[3] = {0, 0, 0};
  void register_face(int ngg, int dim);
};

struct Block {
  int mx = 1, my = 1, mz = 1, ngg = 2, id = 0;
  Array3 x, y, z;  // ngg+1 ghost layers while building, ngg afterwards
  Array3 jac;
  std::array<Array3, 9> metric;
  std::vector<Boundary> boundary;
  std::vector<InnerFace> inner_face;
  Block(int mx_, int my_, int mz_, int ngg_, int id_);
  int64_t n_cells() const { return static_cast<int64_t>(mx) * my * mz; }
  // Central-difference Jacobian and metric (src/Mesh.cpp:259-521).
  void compute_jac_metric(const std::string &case_dir);
  void trim_ghost_layers();

 private:
  bool metric_at(int i, int j, int k);
  void log_negative_jacobian(const std::string &case_dir, int i, int j, int k) const;
};

class Mesh {
 public:
  int dimension = 3;
  int n_block = 0;
  int ngg = 2;
  int64_t n_grid_total = 0;
  std::vector<Block> block;

  Mesh() = default;
  // exact_inner: the ghost grid of every inner face, its tangential ghost
  // rows included, is the neighbour's grid, so that the metrics next to the
  // face are those of the same grid as one block (see DriverOptions)
  explicit Mesh(Parameter &parameter, bool exact_inner = false);
  Block &operator[](size_t i) { return block[i]; }
  const Block &operator[](size_t i) const { return block[i]; }

 private:
  void read_grid(const std::string &case_dir);
  void read_boundary(const std::string &case_dir);
  void read_inner_interface(const std::string &case_dir);
  void scale(double s);
  void init_ghost_grid();
  void init_inner_ghost_grid(int tangential_ghosts = 0);
};

std::string process_file_name(const std::string &stem, int id, const std::string &ext);

}  // namespace ostc
