#include "plt_io.hpp"

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>

#include "text.hpp"

namespace ostc {

namespace {

struct Out {
  std::vector<char> buf;
  void bytes(const void *p, size_t n) {
    const char *c = static_cast<const char *>(p);
    buf.insert(buf.end(), c, c + n);
  }
  void i32(int32_t v) { bytes(&v, 4); }
  void f32(float v) { bytes(&v, 4); }
  void f64(double v) { bytes(&v, 8); }
  // Tecplot strings: one int32 per character and a terminating 0.
  void str(const std::string &s) {
    for (char ch : s) i32(static_cast<int32_t>(ch));
    i32(0);
  }
};

struct In {
  std::vector<char> buf;
  size_t pos = 0;
  bool ok(size_t n) const { return pos + n <= buf.size(); }
  int32_t i32() {
    int32_t v = 0;
    if (ok(4)) std::memcpy(&v, &buf[pos], 4);
    pos += 4;
    return v;
  }
  std::string str() {
    std::string s;
    while (ok(4)) {
      const int32_t c = i32();
      if (static_cast<char>(c) == '\0') break;
      s += static_cast<char>(c);
    }
    return s;
  }
};

// Interior values of component l of a ghosted array, Fortran order.
template <typename F>
void for_interior(const Block &b, F &&f) {
  for (int k = 0; k < b.mz; ++k)
    for (int j = 0; j < b.my; ++j)
      for (int i = 0; i < b.mx; ++i) f(i, j, k);
}

}  // namespace

std::vector<std::string> plt_variable_names(const Species &spec, bool rans) {
  std::vector<std::string> names = {"x", "y", "z", "density", "u", "v", "w", "pressure", "temperature", "mach"};
  if (spec.n_spec > 0) {
    names.resize(10 + spec.n_spec);
    for (const auto &[name, idx] : spec.spec_list) names[10 + idx] = name;
  }
  if (rans) {
    names.emplace_back("tke");
    names.emplace_back("omega");
    names.emplace_back("mut");
  }
  return names;
}

void write_plt(const std::string &path, const std::vector<PltBlockData> &blocks, const Species &spec, bool rans) {
  const auto names = plt_variable_names(spec, rans);
  const int nvar = static_cast<int>(names.size());
  Out o;
  o.bytes("#!TDV112", 8);
  o.i32(1);
  o.i32(0);
  o.str("Solution file");
  o.i32(nvar);
  for (const auto &n : names) o.str(n);
  for (size_t z = 0; z < blocks.size(); ++z) {
    const Block &b = *blocks[z].block;
    o.f32(299.0f);
    o.str("zone " + std::to_string(z));
    o.i32(-1);
    o.i32(-2);
    o.f64(0.0);
    o.i32(-1);
    o.i32(0);
    o.i32(0);
    o.i32(0);
    o.i32(0);
    o.i32(b.mx);
    o.i32(b.my);
    o.i32(b.mz);
    o.i32(0);
  }
  o.f32(357.0f);
  // The header goes out first; then each zone's data header (with the
  // variables' interior min / max) and its data, streamed one k-plane of one
  // variable at a time: interior rows are contiguous in the ghosted layout,
  // so a plane is mz row copies into one reused buffer.
  const auto parent = std::filesystem::path(path).parent_path();
  if (!parent.empty()) std::filesystem::create_directories(parent);
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  if (!f) throw ParameterError("cannot write " + path);
  f.write(o.buf.data(), static_cast<std::streamsize>(o.buf.size()));
  std::vector<double> plane;
  for (const auto &bd : blocks) {
    const Block &b = *bd.block;
    const HostField &F = *bd.field;
    const Extent &e = F.e;
    // the variable arrays of this zone in file order
    std::vector<std::pair<const double *, const Extent *>> vars;
    vars.push_back({b.x.v.data(), &b.x.e});
    vars.push_back({b.y.v.data(), &b.y.e});
    vars.push_back({b.z.v.data(), &b.z.e});
    for (int l = 0; l < 6; ++l) vars.push_back({F.bv.data() + l * e.size(), &e});
    vars.push_back({bd.mach->data(), &e});
    for (int l = 0; l < F.n_scalar; ++l) vars.push_back({F.sv.data() + l * e.size(), &e});
    if (rans) vars.push_back({bd.mut->data(), &e});
    Out z;
    z.f32(299.0f);
    for (int l = 0; l < nvar; ++l) z.i32(2);
    z.i32(0);
    z.i32(0);
    z.i32(-1);
    for (const auto &[ptr, ext] : vars) {
      double lo = ptr[ext->at(0, 0, 0)], hi = lo;
      for (int k = 0; k < b.mz; ++k)
        for (int j = 0; j < b.my; ++j) {
          const double *row = ptr + ext->at(0, j, k);
          for (int i = 0; i < b.mx; ++i) {
            lo = std::min(lo, row[i]);
            hi = std::max(hi, row[i]);
          }
        }
      z.f64(lo);
      z.f64(hi);
    }
    f.write(z.buf.data(), static_cast<std::streamsize>(z.buf.size()));
    plane.resize(static_cast<size_t>(b.mx) * b.my);
    for (const auto &[ptr, ext] : vars)
      for (int k = 0; k < b.mz; ++k) {
        for (int j = 0; j < b.my; ++j)
          std::memcpy(plane.data() + static_cast<size_t>(j) * b.mx, ptr + ext->at(0, j, k), sizeof(double) * b.mx);
        f.write(reinterpret_cast<const char *>(plane.data()), static_cast<std::streamsize>(sizeof(double) * plane.size()));
      }
  }
  if (!f) throw ParameterError("cannot write " + path);
}

bool read_plt_restart(const std::string &path, const Mesh &mesh, const Species &spec, Parameter &parameter,
                      std::vector<HostField> &field) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return false;
  In in;
  in.buf.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  in.pos = 16;  // magic, byte order, file type
  in.str();     // title
  const int nvar = in.i32();
  std::vector<std::string> names(nvar);
  for (auto &n : names) n = in.str();
  // identify_variable_labels, src/Initialize.cuh:217-276
  const int ns = spec.n_spec, n_turb = parameter.get_int("n_turb");
  const bool rans = parameter.get_int("turbulence_method") == 1 && parameter.get_bool("turbulence");
  int has_spec = 0, has_turb = 0;
  std::vector<int> label(nvar, 999);
  for (int v = 0; v < nvar; ++v) {
    const std::string n = upper(names[v]);
    int l = 999;
    if (n == "DENSITY" || n == "ROE" || n == "RHO") l = 0;
    else if (n == "U") l = 1;
    else if (n == "V") l = 2;
    else if (n == "W") l = 3;
    else if (n == "P" || n == "PRESSURE") l = 4;
    else if (n == "T" || n == "TEMPERATURE") l = 5;
    else {
      if (ns > 0)
        for (const auto &[sname, idx] : spec.spec_list)
          if (n == upper(sname)) {
            l = 6 + idx;
            has_spec = 1;
            break;
          }
      if (rans) {
        if (n == "K" || n == "TKE") {
          if (n_turb == 2) l = 6 + ns;
          has_turb = 2;
        } else if (n == "OMEGA") {
          if (n_turb == 2) l = 6 + ns + 1;
          has_turb = 2;
        }
      }
    }
    label[v] = l;
  }
  const int nz = static_cast<int>(mesh.block.size());
  std::vector<int> mx(nz), my(nz), mz(nz);
  for (int z = 0; z < nz; ++z) {
    in.pos += 4;
    in.str();
    in.pos += 36;
    mx[z] = in.i32();
    my[z] = in.i32();
    mz[z] = in.i32();
    in.pos += 4;
  }
  in.pos += 4;  // end-of-header marker
  for (int z = 0; z < nz; ++z) {
    const Block &b = mesh[z];
    if (mx[z] != b.mx || my[z] != b.my || mz[z] != b.mz)
      throw ParameterError("restart file zone " + std::to_string(z) + " does not match the grid");
    in.pos += 4 + 4 * nvar + 12 + 16 * nvar;
    const size_t npt = static_cast<size_t>(b.mx) * b.my * b.mz;
    in.pos += 3 * npt * 8;
    HostField &F = field[z];
    for (int v = 3; v < nvar; ++v) {
      const int l = label[v];
      double *dst = nullptr;
      if (l < 6) dst = F.bv.data() + l * F.e.size();
      else if (l < 6 + ns) dst = F.sv.data() + (l - 6) * F.e.size();
      else if (l < 6 + ns + n_turb && n_turb == has_turb) dst = F.sv.data() + (l - 6) * F.e.size();
      if (dst) {
        if (!in.ok(npt * 8)) throw ParameterError("restart file " + path + " is truncated");
        for_interior(b, [&](int i, int j, int k) {
          std::memcpy(&dst[F.e.at(i, j, k)], &in.buf[in.pos], 8);
          in.pos += 8;
        });
      } else {
        in.pos += npt * 8;
      }
    }
  }
  // Variables the old run did not have start from the default inflow
  // (src/Initialize.cu:45-104).
  if ((ns > 0 && !has_spec) || (rans && has_turb == 0)) {
    Inflow inflow(parameter.get_string("default_init"), spec, parameter);
    for (int z = 0; z < nz; ++z) {
      const Block &b = mesh[z];
      HostField &F = field[z];
      for_interior(b, [&](int i, int j, int k) {
        if (ns > 0 && !has_spec)
          for (int l = 0; l < ns; ++l) F.s(i, j, k, l) = inflow.sv[l];
        if (rans && has_turb == 0)
          for (int l = 0; l < n_turb; ++l) F.s(i, j, k, ns + l) = inflow.sv[ns + l];
      });
    }
  }
  return true;
}

}  // namespace ostc
