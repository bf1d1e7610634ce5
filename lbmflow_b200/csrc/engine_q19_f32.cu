// Engine<19, float>: one (lattice, storage) instantiation per translation
// unit so the kernels of each pair compile in parallel.
#include "engine.cuh"

namespace lbmb {
EngineBase* make_engine_q19_f32(const lbmb_config& c, const uint8_t* solid, const double* wall_u) {
  return new Engine<19, float>(c, solid, wall_u);
}
}  // namespace lbmb
