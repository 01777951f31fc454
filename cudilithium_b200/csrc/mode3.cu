// Explicit instantiation of the plain batched path and the fused engine for Dilithium3 (one translation unit per
// parameter set so the three sets compile in parallel).
#include "engine_impl.cuh"
#include "host_impl.cuh"

namespace cudil {
template struct Impl<3>;
template struct EngineImpl<3>;
}  // namespace cudil
