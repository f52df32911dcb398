// The reference's main (src/main.cu:7-68) written against include/openstc_b200.hpp;
// used by tests/test_cxx_api.py.
//   cxx_driver_api <case> check   the Mesh and the Driver<...> the setup names
//                                 are built (host only); another Driver<...> throws
//   cxx_driver_api <case> run     ostc::api::run: initialize_computation + simulate
#include <cstdio>
#include <cstring>
#include <stdexcept>

#include "openstc_b200.hpp"

using ostc::api::MixtureModel;
using ostc::api::TurbMethod;

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  try {
    ostc::api::Parameter parameter(argv[1]);
    parameter.options.quiet = 1;
    ostc::api::Mesh mesh(parameter);
    std::printf("blocks %d dimension %d cells %lld first %d %d %d\n", mesh.n_block, mesh.dimension,
                static_cast<long long>(mesh.n_grid_total), mesh.block_dims[0][0], mesh.block_dims[0][1],
                mesh.block_dims[0][2]);
    if (std::strcmp(argv[2], "check") == 0) {
      try {
        ostc::api::Driver<MixtureModel::Air, TurbMethod::Laminar> wrong(parameter, mesh);
        std::printf("a Driver of another configuration was accepted\n");
        return 3;
      } catch (const std::invalid_argument &) {
      }
      ostc::api::Driver<MixtureModel::FR, TurbMethod::RANS> driver(parameter, mesh);
      std::printf("ok %d\n", driver.myid);
      return 0;
    }
    return ostc::api::run(parameter, mesh);
  } catch (const std::exception &e) {
    std::printf("error: %s\n", e.what());
    return 1;
  }
}
