// Engine instantiation: mix=2 turb=1 species=9, FP32-bulk / FP64-critical.
#include "engine_impl.cuh"

namespace ostc {
std::unique_ptr<Engine> make_engine_fr9_sst_mixed(const EngineSetup &s) {
  return std::make_unique<EngineT<Cfg<2, 1, 9, true>>>(s);
}
}  // namespace ostc
