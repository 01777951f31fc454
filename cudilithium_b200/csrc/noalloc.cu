// Batched verification that allocates no device memory.
//
// Who needs it: callers that are not allowed to allocate device memory at the point where they
// verify -- for example a service whose device memory is fully reserved up front by a memory
// budget or pool manager, latency-critical verification threads that must not hit a
// cudaMalloc/cudaFree (both can synchronize the device and stall unrelated streams), or plug-in
// hosts that hand out a stream but own every allocation themselves.  cudil_verify needs a
// caller-allocated pool; this entry point instead uses a fixed scratch array that is part of the
// library image, so the caller passes only its inputs and outputs.
//
// Cost and limits:
//  * the array (CUDIL_NOALLOC_SCRATCH_BYTES = 16 MiB) is reserved on every GPU that loads the
//    library, for as long as the library stays loaded;
//  * one call verifies at most 16 MiB / (verify row size) signatures (about 420 Dilithium2
//    signatures of 32-byte messages); larger batches are rejected with CUDIL_ERR_BUDGET;
//  * all calls share the one array: calls whose work overlaps on the GPU (different streams or
//    host threads without ordering between them) race on it and must be serialized by the caller;
//  * the first call on a device looks up the array's device address (cudaGetSymbolAddress) and
//    caches it; make that first call before capturing any stream into a CUDA graph.
// Nothing in the array needs to start at zero: every byte a verify kernel reads is written earlier
// in the same call (inputs by the copies, the rest by the preceding kernels).
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/cudilithium.h"
#include "host_impl.cuh"

namespace cudil {
extern template struct Impl<2>;
extern template struct Impl<3>;
extern template struct Impl<5>;
}  // namespace cudil

namespace {

constexpr size_t kScratchBytes = CUDIL_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

__device__ __align__(256) uint8_t g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
void *g_scratch_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (looked up once per device).
int scratch_for_current_device(uint8_t **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return CUDIL_ERR_CUDA;
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return CUDIL_ERR_CUDA;
        g_scratch_ptr[dev] = p;
    }
    *out = static_cast<uint8_t *>(g_scratch_ptr[dev]);
    return CUDIL_OK;
}

}  // namespace

extern "C" size_t cudil_verify_noalloc_max_batch(int mode, size_t mlen) {
    const size_t row = cudil::align256(cudil_verify_row_bytes(mode, mlen));
    return row ? kScratchBytes / row : 0;
}

extern "C" int cudil_verify_noalloc(int mode, int *ret, const uint8_t *sig, size_t sig_pitch, size_t siglen,
                                    const uint8_t *m, size_t m_pitch, size_t mlen, const uint8_t *pk,
                                    size_t batch_size, void *stream) {
    cudil_params p;
    if (cudil_get_params(mode, &p) != CUDIL_OK) return CUDIL_ERR_INVALID;
    const size_t row = cudil::align256(cudil_verify_row_bytes(mode, mlen));
    if (batch_size > kScratchBytes / row) return CUDIL_ERR_BUDGET;
    if (batch_size == 0) return CUDIL_OK;
    uint8_t *scratch = nullptr;
    // With a wrong siglen cudil_verify sets every ret to -1 without touching the GPU.
    if (siglen == (size_t)p.sig_bytes) {
        const int rc = scratch_for_current_device(&scratch);
        if (rc != CUDIL_OK) return rc;
    }
    return cudil_verify(mode, ret, sig, sig_pitch, siglen, m, m_pitch, mlen, pk, scratch, row, batch_size, stream);
}
