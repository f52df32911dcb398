// Engine instantiation: mix=1 turb=0 species=9.
#include "engine_impl.cuh"

namespace ostc {
std::unique_ptr<Engine> make_engine_mix9_lam(const EngineSetup &s) {
  return std::make_unique<EngineT<Cfg<1, 0, 9>>>(s);
}
}  // namespace ostc
