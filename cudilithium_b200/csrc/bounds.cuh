// Bounds-checked build (compiled with -DCUDIL_BOUNDS_CHECK; `python cudilithium_b200/build.py
// --bounds-check` makes libcudilithium_b200_bc.so).  Device-side index checks on pool rows, attempt
// slots, item indices and key-cache rows: a failing check records its site code in an error word of
// its translation unit (the first failure wins) and returns false, and the caller skips the access.
// Nothing traps, and kernels with block barriers keep every thread on the barrier path.  In the
// normal build every check is the constant true and compiles away.  cudil_bounds_check_status reads
// (and clears) the error words.
#pragma once

#include <cuda_runtime.h>

namespace cudil {

// Site codes recorded by a failing check (nonzero).
enum BoundsSite : unsigned {
    BC_PREHASH_ITEM = 1,   // prehash: order[] entry or key index out of range
    BC_SIGN_SLOT = 2,      // persistent signer: attempt slot / item index out of range
    BC_SIGN_KEY = 3,       // persistent signer: key-cache row index out of range
    BC_VERIFY_KEY = 4,     // persistent verifier: key-cache row index out of range
    BC_STAGE_ITEM = 5,     // plain path stage kernels: exec slot names an item outside the batch
    BC_COPY_ENTRY = 6,     // plain path signature copy: copy-LUT entry out of range
};

#ifdef CUDIL_BOUNDS_CHECK
static __device__ unsigned g_bounds_error;

__device__ __forceinline__ bool bc_ok(bool cond, unsigned site) {
    if (!cond) atomicCAS(&g_bounds_error, 0u, site);
    return cond;
}

// Host: this translation unit's error word (and clear it when reset); 0 = no check failed.
static inline cudaError_t bounds_status_here(unsigned *out, bool reset) {
    unsigned v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_bounds_error, sizeof v);
    if (e == cudaSuccess && reset) {
        const unsigned z = 0;
        e = cudaMemcpyToSymbol(g_bounds_error, &z, sizeof z);
    }
    *out = v;
    return e;
}
constexpr bool kBoundsChecked = true;
#else
__device__ __forceinline__ constexpr bool bc_ok(bool, unsigned) { return true; }
static inline cudaError_t bounds_status_here(unsigned *out, bool) {
    *out = 0;
    return cudaSuccess;
}
constexpr bool kBoundsChecked = false;
#endif

}  // namespace cudil
