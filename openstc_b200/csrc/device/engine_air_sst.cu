// Engine instantiation: mix=0 turb=1 species=0.
#include "engine_impl.cuh"

namespace ostc {
std::unique_ptr<Engine> make_engine_air_sst(const EngineSetup &s) {
  return std::make_unique<EngineT<Cfg<0, 1, 0>>>(s);
}
}  // namespace ostc
