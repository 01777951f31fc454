// Explicit instantiation of the plain batched path and the fused engine for Dilithium5 (one translation unit per
// parameter set so the three sets compile in parallel).
#include "engine_impl.cuh"
#include "host_impl.cuh"

namespace cudil {
template struct Impl<5>;
template struct EngineImpl<5>;
}  // namespace cudil
