// Explicit instantiation of the plain batched path and the fused engine for Dilithium3 (one translation unit per
// parameter set so the three sets compile in parallel).
#include "engine_impl.cuh"
#include "host_impl.cuh"

namespace cudil {
template struct Impl<3>;
template struct EngineImpl<3>;

// Error word of this translation unit's kernels in the bounds-checked build (see bounds.cuh).
cudaError_t bounds_status_mode3(unsigned *out, bool reset) { return bounds_status_here(out, reset); }
}  // namespace cudil
