// Engine factory and error helper.
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "engine.hpp"

namespace ostc {

void cuda_check(int err, const char *what) {
  if (err != cudaSuccess) {
    throw std::runtime_error(std::string("CUDA error in ") + what + ": " +
                             cudaGetErrorString(static_cast<cudaError_t>(err)));
  }
}

std::unique_ptr<Engine> make_engine(const EngineSetup &s) {
  const auto &p = s.params;
  const bool sst = p.turb == 1;
  if (p.turb == 1 && p.rans_model != 2) throw std::runtime_error("only the k-omega SST RANS model is implemented");
  if (s.precision == 1 && (p.mix != 2 || !sst))
    throw std::runtime_error("the FP32-bulk / FP64-critical kernels are built for the finite-rate SST configuration");
  if (p.mix == 0) return sst ? make_engine_air_sst(s) : make_engine_air_lam(s);
  if (p.ns != 9)
    throw std::runtime_error("species engines are instantiated for 9 species; this mechanism has " +
                             std::to_string(p.ns));
  if (s.precision == 1) return make_engine_fr9_sst_mixed(s);
  if (p.mix == 1) return sst ? make_engine_mix9_sst(s) : make_engine_mix9_lam(s);
  return sst ? make_engine_fr9_sst(s) : make_engine_fr9_lam(s);
}

}  // namespace ostc
