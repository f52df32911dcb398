// Engine instantiation: mix=2 turb=1 species=9.
#include "engine_impl.cuh"

namespace ostc {
std::unique_ptr<Engine> make_engine_fr9_sst(const EngineSetup &s) {
  return std::make_unique<EngineT<Cfg<2, 1, 9>>>(s);
}
}  // namespace ostc
