#include "mesh.hpp"

#include <cmath>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <sstream>

namespace ostc {

namespace {
int sgn(int a) { return a < 0 ? -1 : 1; }
}  // namespace

std::string process_file_name(const std::string &stem, int id, const std::string &ext) {
  // fmt "{:>4}": the process id right-aligned in four columns ("grid   0.grd").
  char buf[32];
  std::snprintf(buf, sizeof(buf), "%4d", id);
  return stem + buf + ext;
}

// ---------------------------------------------------------------- faces
void Boundary::register_face(int ngg, int dim) {
  // src/Mesh.cpp:18-35
  for (int i = 0; i < dim; ++i) {
    if (start[i] == end[i]) {
      face = i;
      if (start[i] == 0) direction = -1;
      break;
    }
  }
  for (int i = 0; i < dim; ++i) {
    if (i == face) continue;
    if (end[i] < start[i]) std::swap(end[i], start[i]);
    start[i] -= ngg;
    end[i] += ngg;
  }
  if (dim == 2) {
    start[2] = -ngg;
    end[2] = ngg;
  }
}

void InnerFace::register_face(int ngg, int dim) {
  // src/Mesh.cpp:47-177: 1-based input, a negative tangential range marks the
  // first tangential direction in 3D, and the normal range becomes the face
  // plus its ngg ghost layers.
  for (int i = 0; i < dim; ++i) {
    if (start[i] == end[i]) {
      face = i;
      if (start[i] == 1) direction = -1;
      start[i] -= 1;
      end[i] -= 1;
      break;
    }
  }
  for (int i = 0; i < dim; ++i) {
    if (tstart[i] == tend[i]) {
      target_face = i;
      if (tstart[i] == 1) target_direction = -1;
      tstart[i] -= 1;
      tend[i] -= 1;
      break;
    }
  }
  src_tar[target_face] = -(direction * target_direction) * (face + 1);
  if (dim == 2) {
    const int nf = 1 - face, tnf = 1 - target_face;
    start[nf] = std::abs(start[nf]) - 1;
    end[nf] = std::abs(end[nf]) - 1;
    // The reference indexes the target range with the source's tangential
    // direction here (src/Mesh.cpp:71-72); kept as is.
    tstart[nf] = std::abs(tstart[nf]) - 1;
    tend[nf] = std::abs(tend[nf]) - 1;
    src_tar[tnf] = sgn((tend[tnf] - tstart[tnf]) * (end[nf] - start[nf])) * (nf + 1);
    src_tar[2] = 3;
    start[2] = end[2] = tstart[2] = tend[2] = 0;
  } else {
    int nf = 0, tnf = 0;
    for (int i = 0; i < dim; ++i) {
      if (start[i] < 0) {
        nf = i;
        start[i] = -start[i] - 1;
        end[i] = -end[i] - 1;
        break;
      }
    }
    for (int i = 0; i < dim; ++i) {
      if (tstart[i] < 0) {
        tnf = i;
        tstart[i] = -tstart[i] - 1;
        tend[i] = -tend[i] - 1;
        break;
      }
    }
    src_tar[tnf] = sgn((tend[tnf] - tstart[tnf]) * (end[nf] - start[nf])) * (nf + 1);
    nf = 3 - face - nf;
    tnf = 3 - target_face - tnf;
    start[nf] -= 1;
    end[nf] -= 1;
    tstart[tnf] -= 1;
    tend[tnf] -= 1;
    src_tar[tnf] = sgn((tend[tnf] - tstart[tnf]) * (end[nf] - start[nf])) * (nf + 1);
  }
  start[face] = direction < 0 ? -ngg : end[face];
  end[face] = direction < 0 ? 0 : end[face] + ngg;
  const int sgn_tar = sgn(src_tar[target_face]);
  if (target_direction > 0) {
    tstart[target_face] = sgn_tar > 0 ? tend[target_face] - ngg : tend[target_face];
  } else {
    tstart[target_face] = sgn_tar > 0 ? 0 : ngg;
  }
  for (int i = 0; i < 3; ++i) {
    loop_dir[i] = start[i] <= end[i] ? 1 : -1;
    target_loop_dir[i] = sgn(src_tar[i]);
    src_tar[i] = std::abs(src_tar[i]) - 1;
  }
  for (int i = 0; i < 3; ++i) n_point[i] = std::abs(start[i] - end[i]) + 1;
}

// ---------------------------------------------------------------- block
Block::Block(int mx_, int my_, int mz_, int ngg_, int id_)
    : mx(mx_), my(my_), mz(mz_), ngg(ngg_), id(id_),
      x(mx_, my_, mz_, ngg_ + 1), y(mx_, my_, mz_, ngg_ + 1), z(mx_, my_, mz_, ngg_ + 1),
      jac(mx_, my_, mz_, ngg_) {
  for (auto &m : metric) m = Array3(mx_, my_, mz_, ngg_);
}

bool Block::metric_at(int i, int j, int k) {
  const double dxd1 = (x(i + 1, j, k) - x(i - 1, j, k)) * 0.5, dyd1 = (y(i + 1, j, k) - y(i - 1, j, k)) * 0.5,
               dzd1 = (z(i + 1, j, k) - z(i - 1, j, k)) * 0.5;
  const double dxd2 = (x(i, j + 1, k) - x(i, j - 1, k)) * 0.5, dyd2 = (y(i, j + 1, k) - y(i, j - 1, k)) * 0.5,
               dzd2 = (z(i, j + 1, k) - z(i, j - 1, k)) * 0.5;
  const double dxd3 = (x(i, j, k + 1) - x(i, j, k - 1)) * 0.5, dyd3 = (y(i, j, k + 1) - y(i, j, k - 1)) * 0.5,
               dzd3 = (z(i, j, k + 1) - z(i, j, k - 1)) * 0.5;
  const double J = dxd1 * dyd2 * dzd3 + dxd2 * dyd3 * dzd1 + dxd3 * dyd1 * dzd2 - dxd1 * dyd3 * dzd2 -
                   dxd2 * dyd1 * dzd3 - dxd3 * dyd2 * dzd1;
  if (J <= 0) return false;
  jac(i, j, k) = J;
  metric[0](i, j, k) = (dyd2 * dzd3 - dyd3 * dzd2) / J;
  metric[1](i, j, k) = (dxd3 * dzd2 - dxd2 * dzd3) / J;
  metric[2](i, j, k) = (dxd2 * dyd3 - dxd3 * dyd2) / J;
  metric[3](i, j, k) = (dyd3 * dzd1 - dyd1 * dzd3) / J;
  metric[4](i, j, k) = (dxd1 * dzd3 - dxd3 * dzd1) / J;
  metric[5](i, j, k) = (dxd3 * dyd1 - dxd1 * dyd3) / J;
  metric[6](i, j, k) = (dyd1 * dzd2 - dyd2 * dzd1) / J;
  metric[7](i, j, k) = (dxd2 * dzd1 - dxd1 * dzd2) / J;
  metric[8](i, j, k) = (dxd1 * dyd2 - dxd2 * dyd1) / J;
  return true;
}

void Block::log_negative_jacobian(const std::string &case_dir, int i, int j, int k) const {
  // src/Mesh.cpp:523-532: one log file per block, rewritten at every event.
  const std::filesystem::path dir = std::filesystem::path(case_dir) / "error-log" / "negative-jacobian";
  std::filesystem::create_directories(dir);
  std::ofstream log(dir / ("Process_0-Block_" + std::to_string(id) + ".log"));
  log << "Block " << id << ", I = " << i << "\tJ = " << j << "\tK = " << k << "\n";
}

void Block::compute_jac_metric(const std::string &case_dir) {
  auto copy_from = [&](int i, int j, int k, int si, int sj, int sk) {
    jac(i, j, k) = jac(si, sj, sk);
    for (auto &m : metric) m(i, j, k) = m(si, sj, sk);
  };
  const int kmin = (mz == 1) ? 0 : 1, kmax = (mz == 1) ? 1 : mz - 1;
  for (int i = 1; i < mx - 1; ++i)
    for (int j = 1; j < my - 1; ++j)
      for (int k = kmin; k < kmax; ++k)
        if (!metric_at(i, j, k)) {
          char msg[160];
          std::snprintf(msg, sizeof(msg), "Negative Jacobian from process 0\nBlock %d, index is (%d, %d, %d).", id, i,
                        j, k);
          throw ParameterError(msg);
        }
  for (int i = 1; i < mx - 1; ++i)
    for (int j = 1; j < my - 1; ++j)
      for (int k = 0; k >= -ngg; --k)
        if (!metric_at(i, j, k)) log_negative_jacobian(case_dir, i, j, k), copy_from(i, j, k, i, j, k + 1);
  for (int i = 1; i < mx - 1; ++i)
    for (int j = 1; j < my - 1; ++j)
      for (int k = mz - 1; k < mz + ngg; ++k)
        if (!metric_at(i, j, k)) log_negative_jacobian(case_dir, i, j, k), copy_from(i, j, k, i, j, k - 1);
  for (int i = 1; i < mx - 1; ++i)
    for (int j = 0; j >= -ngg; --j)
      for (int k = -ngg; k < mz + ngg; ++k)
        if (!metric_at(i, j, k)) log_negative_jacobian(case_dir, i, j, k), copy_from(i, j, k, i, j + 1, k);
  for (int i = 1; i < mx - 1; ++i)
    for (int j = my - 1; j < my + ngg; ++j)
      for (int k = -ngg; k < mz + ngg; ++k)
        if (!metric_at(i, j, k)) log_negative_jacobian(case_dir, i, j, k), copy_from(i, j, k, i, j - 1, k);
  for (int i = 0; i >= -ngg; --i)
    for (int j = -ngg; j < my + ngg; ++j)
      for (int k = -ngg; k < mz + ngg; ++k)
        if (!metric_at(i, j, k)) log_negative_jacobian(case_dir, i, j, k), copy_from(i, j, k, i + 1, j, k);
  for (int i = mx - 1; i < mx + ngg; ++i)
    for (int j = -ngg; j < my + ngg; ++j)
      for (int k = -ngg; k < mz + ngg; ++k)
        if (!metric_at(i, j, k)) log_negative_jacobian(case_dir, i, j, k), copy_from(i, j, k, i - 1, j, k);
}

void Block::trim_ghost_layers() {
  for (Array3 *a : {&x, &y, &z}) {
    Array3 t(mx, my, mz, ngg);
    for (int i = -ngg; i < mx + ngg; ++i)
      for (int j = -ngg; j < my + ngg; ++j)
        for (int k = -ngg; k < mz + ngg; ++k) t(i, j, k) = (*a)(i, j, k);
    *a = std::move(t);
  }
}

// ---------------------------------------------------------------- mesh
Mesh::Mesh(Parameter &parameter, bool exact_inner)
    : dimension(parameter.get_int("dimension")), ngg(parameter.get_int("ngg")) {
  const std::string &dir = parameter.case_dir();
  read_grid(dir);
  parameter.set("n_block", n_block);
  read_boundary(dir);
  read_inner_interface(dir);
  const double s = parameter.get_real("gridScale");
  if (std::abs(s - 1.0) > 1e-15) scale(s);
  init_ghost_grid();
  // after the edge and corner completion: the neighbours' own ghost rows
  if (exact_inner) init_inner_ghost_grid(ngg + 1);
  for (auto &b : block) b.compute_jac_metric(dir);
  for (auto &b : block) b.trim_ghost_layers();
}

void Mesh::read_grid(const std::string &case_dir) {
  const std::string path = case_dir + "/input_files/grid/" + process_file_name("grid", 0, ".grd");
  std::ifstream grd(path);
  if (!grd) throw ParameterError("cannot open grid file " + path);
  std::string input;
  std::getline(grd, input);
  n_block = std::stoi(input);
  for (int b = 0; b < n_block; ++b) {
    std::getline(grd, input);
    std::istringstream ls(input);
    int mx = 0, my = 0, mz = 0;
    ls >> mx >> my >> mz;
    if (mx < 3 || my < 3 || mz < 1) throw ParameterError("block " + std::to_string(b) + " is too small");
    block.emplace_back(mx, my, mz, ngg, b);
  }
  if (block.at(0).mz == 1) dimension = 2;
  n_grid_total = 0;
  for (auto &b : block) n_grid_total += b.n_cells();
  for (auto &b : block) {
    for (Array3 *a : {&b.x, &b.y, &b.z})
      for (int k = 0; k < b.mz; ++k)
        for (int j = 0; j < b.my; ++j)
          for (int i = 0; i < b.mx; ++i)
            if (!(grd >> (*a)(i, j, k))) throw ParameterError("grid file " + path + " ended early");
  }
}

void Mesh::read_boundary(const std::string &case_dir) {
  const std::string path = case_dir + "/input_files/boundary_condition/" + process_file_name("boundary", 0, ".txt");
  std::ifstream f(path);
  if (!f) throw ParameterError("cannot open boundary file " + path);
  std::string input;
  for (auto &b : block) {
    std::getline(f, input);
    const int n = std::stoi(input);
    for (int q = 0; q < n; ++q) {
      std::getline(f, input);
      std::istringstream ls(input);
      Boundary bc;
      ls >> bc.start[0] >> bc.end[0] >> bc.start[1] >> bc.end[1] >> bc.start[2] >> bc.end[2] >> bc.label;
      bc.register_face(ngg, dimension);
      b.boundary.push_back(bc);
    }
  }
}

void Mesh::read_inner_interface(const std::string &case_dir) {
  const std::string path = case_dir + "/input_files/boundary_condition/" + process_file_name("inner", 0, ".txt");
  std::ifstream f(path);
  if (!f) throw ParameterError("cannot open inner-face file " + path);
  std::string input;
  std::getline(f, input);
  std::vector<int> n_face(n_block, 0);
  for (int b = 0; b < n_block; ++b) f >> n_face[b];
  std::getline(f, input);
  std::getline(f, input);
  for (int b = 0; b < n_block; ++b) {
    for (int q = 0; q < n_face[b]; ++q) {
      InnerFace fc{};
      int unused = 0, tb = 0;
      std::getline(f, input);
      {
        std::istringstream ls(input);
        ls >> fc.start[0] >> fc.end[0] >> fc.start[1] >> fc.end[1] >> fc.start[2] >> fc.end[2] >> unused;
      }
      std::getline(f, input);
      {
        std::istringstream ls(input);
        ls >> fc.tstart[0] >> fc.tend[0] >> fc.tstart[1] >> fc.tend[1] >> fc.tstart[2] >> fc.tend[2] >> tb;
      }
      fc.target_block = tb - 1;
      fc.face = 0;
      fc.direction = 1;
      fc.target_face = 0;
      fc.target_direction = 1;
      for (int i = 0; i < 3; ++i) {
        fc.src_tar[i] = 0;
        fc.loop_dir[i] = 1;
        fc.target_loop_dir[i] = 1;
      }
      fc.register_face(ngg, dimension);
      if (fc.target_block < 0 || fc.target_block >= n_block)
        throw ParameterError("inner face of block " + std::to_string(b) + " targets a missing block");
      block[b].inner_face.push_back(fc);
    }
  }
}

void Mesh::scale(double s) {
  for (auto &b : block)
    for (Array3 *a : {&b.x, &b.y, &b.z})
      for (auto &v : a->v) v *= s;
}

void Mesh::init_ghost_grid() {
  // src/Mesh.cpp:789-943: mirror through the boundary point, then inner-face
  // copies, then parallelogram completion of edges and corners.
  const int g1 = ngg + 1;
  for (auto &B : block) {
    const int mx = B.mx, my = B.my, mz = B.mz;
    for (int k = 0; k < mz; ++k)
      for (int j = 0; j < my; ++j) {
        for (int i = -1; i >= -g1; --i) {
          B.x(i, j, k) = 2 * B.x(0, j, k) - B.x(-i, j, k);
          B.y(i, j, k) = 2 * B.y(0, j, k) - B.y(-i, j, k);
          B.z(i, j, k) = 2 * B.z(0, j, k) - B.z(-i, j, k);
        }
        for (int i = mx; i < mx + g1; ++i) {
          B.x(i, j, k) = 2 * B.x(mx - 1, j, k) - B.x(2 * (mx - 1) - i, j, k);
          B.y(i, j, k) = 2 * B.y(mx - 1, j, k) - B.y(2 * (mx - 1) - i, j, k);
          B.z(i, j, k) = 2 * B.z(mx - 1, j, k) - B.z(2 * (mx - 1) - i, j, k);
        }
      }
    for (int k = 0; k < mz; ++k)
      for (int i = 0; i < mx; ++i) {
        for (int j = -1; j >= -g1; --j) {
          B.x(i, j, k) = 2 * B.x(i, 0, k) - B.x(i, -j, k);
          B.y(i, j, k) = 2 * B.y(i, 0, k) - B.y(i, -j, k);
          B.z(i, j, k) = 2 * B.z(i, 0, k) - B.z(i, -j, k);
        }
        for (int j = my; j < my + g1; ++j) {
          B.x(i, j, k) = 2 * B.x(i, my - 1, k) - B.x(i, 2 * (my - 1) - j, k);
          B.y(i, j, k) = 2 * B.y(i, my - 1, k) - B.y(i, 2 * (my - 1) - j, k);
          B.z(i, j, k) = 2 * B.z(i, my - 1, k) - B.z(i, 2 * (my - 1) - j, k);
        }
      }
    if (dimension == 3) {
      for (int j = 0; j < my; ++j)
        for (int i = 0; i < mx; ++i) {
          for (int k = -1; k >= -g1; --k) {
            B.x(i, j, k) = 2 * B.x(i, j, 0) - B.x(i, j, -k);
            B.y(i, j, k) = 2 * B.y(i, j, 0) - B.y(i, j, -k);
            B.z(i, j, k) = 2 * B.z(i, j, 0) - B.z(i, j, -k);
          }
          for (int k = mz; k < mz + g1; ++k) {
            B.x(i, j, k) = 2 * B.x(i, j, mz - 1) - B.x(i, j, 2 * (mz - 1) - k);
            B.y(i, j, k) = 2 * B.y(i, j, mz - 1) - B.y(i, j, 2 * (mz - 1) - k);
            B.z(i, j, k) = 2 * B.z(i, j, mz - 1) - B.z(i, j, 2 * (mz - 1) - k);
          }
        }
    } else {
      for (int j = 0; j < my; ++j)
        for (int i = 0; i < mx; ++i) {
          for (int k = -1; k >= -g1; --k) {
            B.x(i, j, k) = B.x(i, j, 0);
            B.y(i, j, k) = B.y(i, j, 0);
            B.z(i, j, k) = B.z(i, j, 0) + k;
          }
          for (int k = mz; k < mz + g1; ++k) {
            B.x(i, j, k) = B.x(i, j, mz - 1);
            B.y(i, j, k) = B.y(i, j, mz - 1);
            B.z(i, j, k) = B.z(i, j, mz - 1) + k - mz + 1;
          }
        }
    }
  }
  init_inner_ghost_grid();
  for (auto &B : block) {
    const int mx = B.mx, my = B.my, mz = B.mz;
    Array3 *xyz[3] = {&B.x, &B.y, &B.z};
    for (int i = 1; i <= g1; ++i)
      for (int j = 1; j <= g1; ++j)
        for (int k = 0; k < mz; ++k) {
          const int i1 = -i, j1 = -j, i2 = mx - 1 + i, j2 = my - 1 + j;
          for (Array3 *a : xyz) {
            Array3 &A = *a;
            A(i1, j1, k) = A(i1, 0, k) + A(0, j1, k) - A(0, 0, k);
            A(i2, j2, k) = A(i2, my - 1, k) + A(mx - 1, j2, k) - A(mx - 1, my - 1, k);
            A(i1, j2, k) = A(i1, my - 1, k) + A(0, j2, k) - A(0, my - 1, k);
            A(i2, j1, k) = A(i2, 0, k) + A(mx - 1, j1, k) - A(mx - 1, 0, k);
          }
        }
    for (int i = 1; i <= g1; ++i)
      for (int j = 0; j < my; ++j)
        for (int k = 1; k <= g1; ++k) {
          const int i1 = -i, k1 = -k, i2 = mx - 1 + i, k2 = mz - 1 + k;
          for (Array3 *a : xyz) {
            Array3 &A = *a;
            A(i1, j, k1) = A(i1, j, 0) + A(0, j, k1) - A(0, j, 0);
            A(i2, j, k2) = A(i2, j, mz - 1) + A(mx - 1, j, k2) - A(mx - 1, j, mz - 1);
            A(i1, j, k2) = A(i1, j, mz - 1) + A(0, j, k2) - A(0, j, mz - 1);
            A(i2, j, k1) = A(i2, j, 0) + A(mx - 1, j, k1) - A(mx - 1, j, 0);
          }
        }
    for (int i = -g1; i <= mx + ngg; ++i)
      for (int j = 1; j <= g1; ++j)
        for (int k = 1; k <= g1; ++k) {
          const int j1 = -j, k1 = -k, j2 = my - 1 + j, k2 = mz - 1 + k;
          for (Array3 *a : xyz) {
            Array3 &A = *a;
            A(i, j1, k1) = A(i, j1, 0) + A(i, 0, k1) - A(i, 0, 0);
            A(i, j2, k2) = A(i, j2, mz - 1) + A(i, my - 1, k2) - A(i, my - 1, mz - 1);
            A(i, j1, k2) = A(i, j1, mz - 1) + A(i, 0, k2) - A(i, 0, mz - 1);
            A(i, j2, k1) = A(i, j2, 0) + A(i, my - 1, k1) - A(i, my - 1, 0);
          }
        }
  }
}

void Mesh::init_inner_ghost_grid(int tangential_ghosts) {
  // src/Mesh.cpp:945-993.  tangential_ghosts > 0 extends the copy by that many
  // rows past the face's tangential ends (exact inner faces; faces that cover
  // the whole block face in the same orientation as the neighbour's).
  for (auto &B : block) {
    for (const auto &fc : B.inner_face) {
      const Block &N = block[fc.target_block];
      int lo[3] = {fc.start[0], fc.start[1], fc.start[2]};
      int hi[3] = {fc.end[0], fc.end[1], fc.end[2]};
      int tlo[3] = {fc.tstart[0], fc.tstart[1], fc.tstart[2]};
      const int shift = fc.direction < 0 ? -1 : 1;
      lo[fc.face] += shift;
      hi[fc.face] += shift;
      tlo[fc.target_face] += fc.target_direction > 0 ? -1 : 1;
      for (int q = 0; q < 3 && tangential_ghosts > 0; ++q) {
        if (q == fc.face || lo[q] == hi[q]) continue;
        int t = 0;  // the target direction that runs along this one (src_tar: target -> source)
        while (t < 2 && fc.src_tar[t] != q) ++t;
        if (fc.loop_dir[q] < 0 || fc.target_loop_dir[t] < 0)
          throw ParameterError("exact inner faces need faces oriented as their neighbours'");
        lo[q] -= tangential_ghosts;
        hi[q] += tangential_ghosts;
        tlo[t] -= tangential_ghosts;
      }
      int d[3];
      for (int i1 = lo[0]; fc.loop_dir[0] * (i1 - hi[0]) != 1; i1 += fc.loop_dir[0]) {
        d[0] = i1 - lo[0];
        for (int j1 = lo[1]; fc.loop_dir[1] * (j1 - hi[1]) != 1; j1 += fc.loop_dir[1]) {
          d[1] = j1 - lo[1];
          for (int k1 = lo[2]; fc.loop_dir[2] * (k1 - hi[2]) != 1; k1 += fc.loop_dir[2]) {
            d[2] = k1 - lo[2];
            const int i2 = tlo[0] + fc.target_loop_dir[0] * d[fc.src_tar[0]];
            const int j2 = tlo[1] + fc.target_loop_dir[1] * d[fc.src_tar[1]];
            const int k2 = tlo[2] + fc.target_loop_dir[2] * d[fc.src_tar[2]];
            B.x(i1, j1, k1) = N.x(i2, j2, k2);
            B.y(i1, j1, k1) = N.y(i2, j2, k2);
            B.z(i1, j1, k1) = N.z(i2, j2, k2);
          }
        }
      }
    }
  }
}

}  // namespace ostc
