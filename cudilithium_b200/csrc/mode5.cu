// Explicit instantiation of the plain batched path and the fused engine for Dilithium5 (one translation unit per
// parameter set so the three sets compile in parallel).
#include "engine_impl.cuh"
#include "host_impl.cuh"

namespace cudil {
template struct Impl<5>;
template struct EngineImpl<5>;

// Error word of this translation unit's kernels in the bounds-checked build (see bounds.cuh).
cudaError_t bounds_status_mode5(unsigned *out, bool reset) { return bounds_status_here(out, reset); }
}  // namespace cudil
