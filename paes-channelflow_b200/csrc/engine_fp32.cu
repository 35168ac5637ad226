// Mixed form of the engine: FP32 padded-grid transforms, advection and SGS;
// FP64 pressure solve, mean modes and reductions.
#include "les_engine.cuh"

namespace les {
cudaError_t upload_twiddles_engine_fp32() { return upload_tu_twiddles(); }
EngineBase* make_engine_fp32(const les_config& c) { return new Engine<float>(c); }
}  // namespace les
