// Explicit instantiation of the plain batched path and the fused engine for Dilithium2 (one translation unit per
// parameter set so the three sets compile in parallel).
#include "engine_impl.cuh"
#include "host_impl.cuh"

namespace cudil {
template struct Impl<2>;
template struct EngineImpl<2>;
}  // namespace cudil
