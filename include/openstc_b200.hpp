/* openstc_b200.hpp -- the library's C++ face in the shape of the reference's
   own: Parameter, Mesh, then Driver<MixtureModel, TurbMethod>(Parameter &,
   Mesh &) with initialize_computation() and simulate(), as main builds them
   (src/Driver.cuh:12-46, src/main.cu:7-68, src/Define.h:14-27).  Header only,
   over the C ABI of openstc_b200.h; link libopenstc_b200.so.

   The reference's main, rewritten against this header:

     #include "openstc_b200.hpp"
     int main() {
       ostc::api::Parameter parameter;              // ./input_files/setup/...
       ostc::api::Mesh mesh(parameter);             // ./input_files/grid/...
       return ostc::api::run(parameter, mesh);      // picks Driver<mix, turb>
     }

   Differences, each deliberate: Parameter takes the case directory (default
   "."), where the reference's reads the current directory through its MPI
   object; the template arguments are checked against the setup files and a
   mismatch throws (the reference's main picks them from the same flags);
   errors of the library throw std::runtime_error with the library's message
   where the reference calls MPI_Abort. */
#ifndef OPENSTC_B200_HPP
#define OPENSTC_B200_HPP

#include <array>
#include <cstdint>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "openstc_b200.h"

namespace ostc {
namespace api {

enum class TurbMethod { Laminar, RANS, LES };          /* src/Define.h:14-20 */
enum class MixtureModel { Air, Mixture, FR, FL };      /* src/Define.h:22-27 */

inline void check(int status) {
  if (status < 0) throw std::runtime_error(ostc_last_error());
}

/* The setup of a case directory (input_files/setup/*.txt are read when the
   Mesh is built) and the options the library adds: device, precision, exact
   inner faces, screen output. */
struct Parameter {
  explicit Parameter(std::string case_dir = ".") : case_dir(std::move(case_dir)) {
    options.device = 0;
    options.quiet = 0;
    options.precision = 0;
    options.exact_inner = 0;
    options.wall_distance = 0;
  }
  std::string case_dir;
  ostc_options options;
};

/* The grid blocks of the case (input_files/grid and boundary_condition);
   building it reads every input file of the case on the host, no GPU work. */
class Mesh {
 public:
  explicit Mesh(Parameter &parameter) {
    ostc_driver *h = nullptr;
    check(ostc_driver_create(parameter.case_dir.c_str(), &parameter.options, &h));
    handle_.reset(h, [](ostc_driver *p) { ostc_driver_destroy(p); });
    ostc_info info;
    check(ostc_driver_info(h, &info));
    n_block = info.n_block;
    dimension = info.dimension;
    ngg = info.ngg;
    n_grid_total = info.n_grid_total;
    for (int b = 0; b < n_block; ++b) {
      std::array<int, 3> d{};
      check(ostc_driver_block_dims(h, b, d.data()));
      block_dims.push_back(d);
    }
  }
  int n_block = 0, dimension = 3, ngg = 2;
  int64_t n_grid_total = 0;
  std::vector<std::array<int, 3>> block_dims;  /* mx, my, mz */
  const std::shared_ptr<ostc_driver> &handle() const { return handle_; }

 private:
  std::shared_ptr<ostc_driver> handle_;
};

template <MixtureModel mix_model, TurbMethod turb_method>
class Driver {
  static_assert(mix_model != MixtureModel::FL, "the flamelet model is not on this path");
  static_assert(turb_method != TurbMethod::LES, "LES is not on this path");

 public:
  /* src/Driver.cu:14-40 */
  Driver(Parameter &parameter_, Mesh &mesh_) : mesh(mesh_), parameter(parameter_), h_(mesh_.handle()) {
    ostc_info info;
    check(ostc_driver_info(h_.get(), &info));
    const int want_mix = mix_model == MixtureModel::Air ? 0 : (mix_model == MixtureModel::Mixture ? 1 : 2);
    const int want_rans = turb_method == TurbMethod::RANS ? 1 : 0;
    if (info.mix != want_mix || info.rans != want_rans)
      throw std::invalid_argument("the case's setup files select another Driver<MixtureModel, TurbMethod>");
  }

  /* src/Driver.cu:44-104 */
  void initialize_computation() { check(ostc_driver_initialize(h_.get())); }

  /* src/Driver.cu:107-289: the steady loop with history.dat, the residual
     files and output/field/flowfield.plt */
  void simulate() {
    check(ostc_driver_simulate(h_.get()));
    check(ostc_driver_residual(h_.get(), res.data()));
    std::ifstream scale(parameter.case_dir + "/output/message/residual_scale.txt");
    for (double &s : res_scale)
      if (!(scale >> s)) break;
  }

  /* The reference's Field arrays of block b (field: ostc_field_id), in its
     column-major layout with ghost layers. */
  std::vector<double> field(int block, int field_id) const {
    int g = 0, nc = 0;
    check(ostc_field_layout(h_.get(), field_id, &g, &nc));
    const auto &d = mesh.block_dims.at(block);
    const int64_t n = static_cast<int64_t>(d[0] + 2 * g) * (d[1] + 2 * g) * (d[2] + 2 * g) * nc;
    std::vector<double> out(static_cast<size_t>(n));
    check(ostc_driver_get_field(h_.get(), block, field_id, out.data(), n));
    return out;
  }

  ostc_driver *handle() const { return h_.get(); }

  int myid = 0;
  const Mesh &mesh;
  const Parameter &parameter;
  std::array<double, 4> res{1, 1, 1, 1};
  std::array<double, 4> res_scale{1, 1, 1, 1};

 private:
  std::shared_ptr<ostc_driver> h_;
};

/* The configuration choice of src/main.cu:22-64: the Driver the setup files
   name, initialised and run.  Returns 0. */
inline int run(Parameter &parameter, Mesh &mesh) {
  ostc_info info;
  check(ostc_driver_info(mesh.handle().get(), &info));
  auto go = [&](auto &&driver) {
    driver.initialize_computation();
    driver.simulate();
    return 0;
  };
  if (info.mix == 2)
    return info.rans ? go(Driver<MixtureModel::FR, TurbMethod::RANS>(parameter, mesh))
                     : go(Driver<MixtureModel::FR, TurbMethod::Laminar>(parameter, mesh));
  if (info.mix == 1)
    return info.rans ? go(Driver<MixtureModel::Mixture, TurbMethod::RANS>(parameter, mesh))
                     : go(Driver<MixtureModel::Mixture, TurbMethod::Laminar>(parameter, mesh));
  return info.rans ? go(Driver<MixtureModel::Air, TurbMethod::RANS>(parameter, mesh))
                   : go(Driver<MixtureModel::Air, TurbMethod::Laminar>(parameter, mesh));
}

}  // namespace api
}  // namespace ostc

#endif
