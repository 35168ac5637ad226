// Plain FP64 form of the engine (one translation unit per precision so the
// templates compile in parallel).
#include "les_engine.cuh"

namespace les {
cudaError_t upload_twiddles_engine_fp64() { return upload_tu_twiddles(); }
EngineBase* make_engine_fp64(const les_config& c) { return new Engine<double>(c); }
}  // namespace les
