// Explicit instantiation of the plain batched path for Dilithium2 (one translation unit per
// parameter set so the three sets compile in parallel).
#include "host_impl.cuh"

namespace cudil {
template struct Impl<2>;
}  // namespace cudil
