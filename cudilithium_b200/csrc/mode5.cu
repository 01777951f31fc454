// Explicit instantiation of the plain batched path for Dilithium5 (one translation unit per
// parameter set so the three sets compile in parallel).
#include "host_impl.cuh"

namespace cudil {
template struct Impl<5>;
}  // namespace cudil
