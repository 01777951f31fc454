// extern "C" boundary of the fused engine (run-time parameter-set dispatch).
#include <new>

#include <cuda_runtime.h>

#include "../../include/cudilithium.h"
#include "engine_impl.cuh"

namespace cudil {
extern template struct EngineImpl<2>;
extern template struct EngineImpl<3>;
extern template struct EngineImpl<5>;
}  // namespace cudil

using namespace cudil;

static_assert(kNonceExhausted == CUDIL_NONCE_EXHAUSTED && kNonceLimit == CUDIL_ENGINE_NONCE_LIMIT &&
                  kLockSpinLimit == CUDIL_ENGINE_LOCK_SPINS && kAsyncIdleLimit == CUDIL_ENGINE_IDLE_POLLS,
              "engine bounds in the C header");

struct cudil_engine {
    EngineBase *impl;
};

#define CUDIL_ENGINE_DISPATCH(e, call)                                  \
    do {                                                                \
        if (!(e) || !(e)->impl) return CUDIL_ERR_INVALID;               \
        switch ((e)->impl->mode) {                                      \
            case 2: {                                                   \
                auto *x = static_cast<EngineImpl<2> *>((e)->impl);      \
                return x->call;                                         \
            }                                                           \
            case 3: {                                                   \
                auto *x = static_cast<EngineImpl<3> *>((e)->impl);      \
                return x->call;                                         \
            }                                                           \
            case 5: {                                                   \
                auto *x = static_cast<EngineImpl<5> *>((e)->impl);      \
                return x->call;                                         \
            }                                                           \
            default:                                                    \
                return CUDIL_ERR_INVALID;                               \
        }                                                               \
    } while (0)

template <int MODE>
static int create_impl(cudil_engine **out, size_t max_keys, size_t max_items, int threads, size_t budget) {
    auto *impl = new (std::nothrow) EngineImpl<MODE>();
    if (!impl) return CUDIL_ERR_INVALID;
    const int rc = impl->create(max_keys, max_items, threads, budget);
    if (rc != CUDIL_OK) {
        delete impl;
        return rc;
    }
    *out = new (std::nothrow) cudil_engine{impl};
    if (!*out) {
        delete impl;
        return CUDIL_ERR_INVALID;
    }
    return CUDIL_OK;
}

extern "C" {

int cudil_engine_create(cudil_engine **out, int mode, size_t max_keys, size_t max_items, int threads_per_block,
                        size_t device_budget_bytes) {
    if (!out) return CUDIL_ERR_INVALID;
    *out = nullptr;
    if (threads_per_block == 0) threads_per_block = 256;
    switch (mode) {
        case 2: return create_impl<2>(out, max_keys, max_items, threads_per_block, device_budget_bytes);
        case 3: return create_impl<3>(out, max_keys, max_items, threads_per_block, device_budget_bytes);
        case 5: return create_impl<5>(out, max_keys, max_items, threads_per_block, device_budget_bytes);
        default: return CUDIL_ERR_INVALID;
    }
}

int cudil_engine_destroy(cudil_engine *e) {
    if (!e) return CUDIL_ERR_INVALID;
    cudaDeviceSynchronize();
    delete e->impl;
    delete e;
    return CUDIL_OK;
}

size_t cudil_engine_device_bytes(const cudil_engine *e) { return (e && e->impl) ? e->impl->device_bytes : 0; }

int cudil_engine_set_secret_keys(cudil_engine *e, const uint8_t *d_sk, size_t nkeys, void *stream) {
    CUDIL_ENGINE_DISPATCH(e, set_secret_keys(d_sk, nkeys, (cudaStream_t)stream));
}

int cudil_engine_update_secret_keys(cudil_engine *e, const uint8_t *d_sk, size_t first, size_t nkeys, void *stream) {
    CUDIL_ENGINE_DISPATCH(e, update_secret_keys(d_sk, first, nkeys, (cudaStream_t)stream));
}

int cudil_engine_set_public_keys(cudil_engine *e, const uint8_t *d_pk, size_t nkeys, void *stream) {
    CUDIL_ENGINE_DISPATCH(e, set_public_keys(d_pk, nkeys, (cudaStream_t)stream));
}

int cudil_engine_sign(cudil_engine *e, uint8_t *d_sig, const uint8_t *d_msgs, size_t msgs_bytes,
                      const unsigned long long *offsets, const uint32_t *mlens, const uint32_t *key_idx, size_t n,
                      void *stream) {
    CUDIL_ENGINE_DISPATCH(e, sign(d_sig, d_msgs, msgs_bytes, offsets, mlens, key_idx, n, (cudaStream_t)stream));
}

int cudil_engine_sign_randomized(cudil_engine *e, uint8_t *d_sig, const uint8_t *d_msgs, size_t msgs_bytes,
                                 const unsigned long long *offsets, const uint32_t *mlens, const uint32_t *key_idx,
                                 const uint8_t *d_rhoprime, size_t n, void *stream) {
    if (!d_rhoprime && n) return CUDIL_ERR_INVALID;
    CUDIL_ENGINE_DISPATCH(e, sign(d_sig, d_msgs, msgs_bytes, offsets, mlens, key_idx, n, (cudaStream_t)stream, d_rhoprime));
}

int cudil_engine_sign_seeded(cudil_engine *e, uint8_t *d_sig, const uint8_t *d_msgs, size_t msgs_bytes,
                             const unsigned long long *offsets, const uint32_t *mlens, const uint32_t *key_idx,
                             const uint8_t *rho_seed, unsigned long long rho_counter, size_t n, void *stream) {
    if (!rho_seed && n) return CUDIL_ERR_INVALID;
    CUDIL_ENGINE_DISPATCH(e, sign(d_sig, d_msgs, msgs_bytes, offsets, mlens, key_idx, n, (cudaStream_t)stream, nullptr,
                                  rho_seed, rho_counter));
}

int cudil_engine_verify(cudil_engine *e, int *d_ret, const uint8_t *d_sig, const uint8_t *d_msgs, size_t msgs_bytes,
                        const unsigned long long *offsets, const uint32_t *mlens, const uint32_t *key_idx, size_t n,
                        void *stream) {
    CUDIL_ENGINE_DISPATCH(e, verify(d_ret, d_sig, d_msgs, msgs_bytes, offsets, mlens, key_idx, n, (cudaStream_t)stream));
}

int cudil_engine_last_status(const cudil_engine *e, unsigned long long *attempts, unsigned *error) {
    if (!e || !e->impl) return CUDIL_ERR_INVALID;
    const FusedQueue *s = e->impl->h_status;
    if (attempts) *attempts = s->attempts;
    if (error) *error = s->error;
    return s->error ? CUDIL_ERR_TIMEOUT : CUDIL_OK;
}

int cudil_engine_last_work(const cudil_engine *e, unsigned long long *attempts, unsigned long long *reject_intt) {
    if (!e || !e->impl) return CUDIL_ERR_INVALID;
    if (attempts) *attempts = e->impl->h_status->attempts;
    if (reject_intt) *reject_intt = e->impl->h_status->intt;
    return CUDIL_OK;
}

int cudil_engine_last_phases(const cudil_engine *e, unsigned long long cycles[4], unsigned *iterations) {
    if (!e || !e->impl) return CUDIL_ERR_INVALID;
    for (int i = 0; i < 4; ++i) cycles[i] = e->impl->h_status->cyc[i];
    if (iterations) *iterations = e->impl->h_status->iters;
    return CUDIL_OK;
}

int cudil_engine_attach_keys(cudil_engine *e, const cudil_engine *src) {
    if (!src || !src->impl) return CUDIL_ERR_INVALID;
    CUDIL_ENGINE_DISPATCH(e, attach_keys(src->impl));
}

int cudil_engine_set_spec_slots(cudil_engine *e, unsigned spec_slots) { CUDIL_ENGINE_DISPATCH(e, set_spec_slots(spec_slots)); }

int cudil_engine_last_jobs(const cudil_engine *e, unsigned long long out[12]) {
    if (!e || !e->impl || !out) return CUDIL_ERR_INVALID;
    for (int i = 0; i < 12; ++i) out[i] = e->impl->h_status->jobs[i];
    return CUDIL_OK;
}

int cudil_engine_set_sign_kernel(cudil_engine *e, int variant) { CUDIL_ENGINE_DISPATCH(e, set_sign_kernel(variant)); }

int cudil_engine_set_limits(cudil_engine *e, unsigned nonce_limit, unsigned lock_spins, unsigned idle_polls) {
    CUDIL_ENGINE_DISPATCH(e, set_limits(nonce_limit, lock_spins, idle_polls));
}

int cudil_engine_last_nonces(cudil_engine *e, unsigned *out, size_t n, void *stream) {
    CUDIL_ENGINE_DISPATCH(e, last_nonces(out, n, (cudaStream_t)stream));
}

int cudil_engine_set_large_batch(cudil_engine *e, size_t min_items, int variant, unsigned spec_slots) {
    CUDIL_ENGINE_DISPATCH(e, set_large_batch(min_items, variant, spec_slots));
}

int cudil_engine_info(const cudil_engine *e, int *mode, int *threads, int *sign_blocks, int *verify_blocks) {
    if (!e || !e->impl) return CUDIL_ERR_INVALID;
    if (mode) *mode = e->impl->mode;
    if (threads) *threads = e->impl->threads;
    if (sign_blocks) {
        const EngineBase *b = e->impl;
        *sign_blocks = b->sign_kernel == 0                        ? b->sign_grid
                       : b->sign_kernel == EngineBase::kWideVariant ? b->wide_grid
                                                                     : b->async_grid[b->sign_kernel - 1];
    }
    if (verify_blocks) *verify_blocks = e->impl->verify_grid;
    return CUDIL_OK;
}

}  // extern "C"
