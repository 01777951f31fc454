// Host side of the fused engine: device buffers sized once at creation, per-key caches, and the
// graph that runs a whole signing (or verification) batch on the device with one launch:
//   [k_fused_init] -> [k_fused_prehash] -> [k_fused_sign]       (sign)
//   [k_fused_init] -> [k_fused_verify_prehash] -> [k_fused_verify] (verify)
// The batch size travels in device memory (FusedQueue::n), so one instantiated graph serves every
// batch size up to the engine's capacity; only the per-item metadata upload precedes the launch.
#pragma once

#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include <cuda_runtime.h>

#include "fused_kernels.cuh"
#include "fused_sign_async.cuh"
#include "host_impl.cuh"
#include "profiling.cuh"

namespace cudil {

struct EngineBase {
    int mode = 0, threads = 0, device = 0, sm_count = 0;
    size_t max_keys = 0, max_items = 0;
    size_t n_sk = 0, n_pk = 0;
    uint8_t *sk_cache = nullptr, *pk_cache = nullptr;
    size_t sk_pitch = 0, pk_pitch = 0;
    uint8_t *items = nullptr;       // max_items * 128
    unsigned *best = nullptr, *locks = nullptr, *next_nonce = nullptr, *inflight = nullptr;
    unsigned spec_slots = 0;  // signer's target of attempts in flight (0 = default for the grid)
    // bounds of the signer's device-side loops (FusedSignArgs)
    unsigned nonce_limit = kNonceLimit, lock_spins = kLockSpinLimit, idle_polls = kAsyncIdleLimit;
    size_t last_n = 0;  // items of the last signing batch
    FusedQueue *q = nullptr;
    // metadata (device) and its pinned staging
    unsigned *d_key = nullptr, *d_mlen = nullptr, *d_order = nullptr;
    unsigned long long *d_off = nullptr;
    uint8_t *h_stage = nullptr;     // [FusedQueue | key | mlen | order | off]
    FusedQueue *h_status = nullptr; // D2H copy of the queue after a batch
    cudaEvent_t stage_ev = nullptr; // recorded after a batch's metadata upload from h_stage
    // key-cache builds run their independent kernels on a side stream too (fork / join events)
    cudaStream_t side = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    bool stage_pending = false;
    uint8_t *scratch = nullptr;
    size_t scratch_bytes = 0;
    int sign_grid = 0, verify_grid = 0, prehash_grid = 0;
    size_t sign_smem = 0, verify_smem = 0;
    // signer kernel: 0 = phased k_fused_sign (block-wide Keccak / NTT phases) with the engine's
    // block size; 1..4 = asynchronous k_fused_sign_async with (threads, slots) per block of
    // (256, 64), (512, 128), (640, 160), (768, 192); 5 = phased with one wide block per SM (512
    // threads, 384 for Dilithium5, whose wider phase buffers allow no more)
    int sign_kernel = 0;
    static constexpr int kAsyncVariants = 4;  // (threads, slots) = (256, 64), (512, 128), (640, 160), (768, 192)
    static constexpr int kWideVariant = kAsyncVariants + 1;
    int async_grid[kAsyncVariants] = {0, 0, 0, 0};
    size_t async_smem[kAsyncVariants] = {0, 0, 0, 0};
    int wide_grid = 0;
    size_t wide_smem = 0;
    // instantiated graphs, keyed by the output / message buffers they were captured with
    cudaGraphExec_t g_sign = nullptr, g_verify = nullptr;
    const void *g_sign_key[3] = {nullptr, nullptr, nullptr}, *g_verify_key[2] = {nullptr, nullptr};
    // Batches of at least large_min_items items (0 = never) sign with large_kernel / large_spec
    // through a graph of their own; smaller ones with sign_kernel / spec_slots.
    size_t large_min_items = 0;
    int large_kernel = 0;
    unsigned large_spec = 0;
    cudaGraphExec_t g_sign_large = nullptr;
    const void *g_sign_large_key[3] = {nullptr, nullptr, nullptr};
    cudaStream_t g_sign_stream = nullptr, g_verify_stream = nullptr;
    size_t device_bytes = 0;
    bool owns_cache = true;  // false when the key caches belong to another engine (attach_keys)
    const EngineBase *key_src = nullptr;  // that engine: its key rows are read as they stand at each call
    virtual ~EngineBase() = default;
};

template <int MODE>
struct EngineImpl : EngineBase {
    using PM = P<MODE>;
    using C = Cache<MODE>;

    // pinned staging: [FusedQueue, padded to 64 bytes | key | mlen | order | off]
    static constexpr size_t kStageHead = (sizeof(FusedQueue) + 63) / 64 * 64;
    static size_t stage_bytes(size_t max_items) {
        return kStageHead + max_items * (3 * sizeof(unsigned) + sizeof(unsigned long long));
    }

    template <int T>
    static int grid_for(const void *fn, size_t smem, int sm_count) {
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, T, smem) != cudaSuccess || per_sm < 1) return 0;
        return per_sm * sm_count;
    }

    // Device bytes the engine needs (the admission budget checks this before allocating).
    size_t required_bytes(size_t max_keys, size_t max_items) const {
        return max_keys * (align256(C::SK_ROW) + align256(C::PK_ROW)) + max_items * (C::ITEM_BYTES + 4 * sizeof(unsigned)) +
               stage_bytes(max_items) + sizeof(FusedQueue) + scratch_for(max_items);
    }
    // attempt slots of the largest signer variant, or the verifier's per-signature slots
    size_t scratch_for(size_t max_items) const {
        if (max_items == 0) return 0;
        size_t b = std::max((size_t)sign_grid * 2 * threads * C::SLOT, (size_t)verify_grid * threads * C::VSLOT);
        static constexpr int slots[kAsyncVariants] = {64, 128, 160, 192};
        for (int v = 0; v < kAsyncVariants; ++v) b = std::max(b, (size_t)async_grid[v] * slots[v] * C::SLOT);
        b = std::max(b, (size_t)wide_grid * 2 * kWideThreads * C::SLOT);
        return b;
    }

    static constexpr int kWideThreads = (MODE == 5) ? 384 : 512;

    int configure_wide() {
        wide_smem = FusedSignSmem<MODE, kWideThreads>::BYTES;
        if (cudaFuncSetAttribute(k_fused_sign<MODE, kWideThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)wide_smem) != cudaSuccess)
            return ::cudil::cudil_record_cuda_error(cudaGetLastError(), __FILE__, __LINE__);
        wide_grid = grid_for<kWideThreads>((const void *)k_fused_sign<MODE, kWideThreads>, wide_smem, sm_count);
        return wide_grid > 0 ? CUDIL_OK : cudil_record_cuda_error(cudaErrorInvalidConfiguration, __FILE__, __LINE__);
    }

    template <int T, int S>
    int configure_async_one(int v) {
        async_smem[v] = AsyncSignSmem<MODE, T, S>::BYTES;
        if (cudaFuncSetAttribute(k_fused_sign_async<MODE, T, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)async_smem[v]) != cudaSuccess)
            return ::cudil::cudil_record_cuda_error(cudaGetLastError(), __FILE__, __LINE__);
        async_grid[v] = grid_for<T>((const void *)k_fused_sign_async<MODE, T, S>, async_smem[v], sm_count);
        return async_grid[v] > 0 ? CUDIL_OK : cudil_record_cuda_error(cudaErrorInvalidConfiguration, __FILE__, __LINE__);
    }

    int configure_async() {
        int rc = configure_async_one<256, 64>(0);
        if (!rc) rc = configure_async_one<512, 128>(1);
        if (!rc) rc = configure_async_one<640, 160>(2);
        if (!rc) rc = configure_async_one<768, 192>(3);
        return rc;
    }

    template <int T>
    int configure() {
        sign_smem = FusedSignSmem<MODE, T>::BYTES;
        verify_smem = FusedVerifySmem<MODE, T>::BYTES;
        if (cudaFuncSetAttribute(k_fused_sign<MODE, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sign_smem) != cudaSuccess ||
            cudaFuncSetAttribute(k_fused_verify<MODE, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)verify_smem) != cudaSuccess)
            return ::cudil::cudil_record_cuda_error(cudaGetLastError(), __FILE__, __LINE__);
        sign_grid = grid_for<T>((const void *)k_fused_sign<MODE, T>, sign_smem, sm_count);
        verify_grid = grid_for<T>((const void *)k_fused_verify<MODE, T>, verify_smem, sm_count);
        return (sign_grid > 0 && verify_grid > 0) ? CUDIL_OK : cudil_record_cuda_error(cudaErrorInvalidConfiguration, __FILE__, __LINE__);
    }

    int create(size_t mk, size_t mi, int thr, size_t budget) {
        mode = MODE;
        max_keys = mk;
        max_items = mi;
        threads = thr;
        // mk == 0: caches attached later; mi == 0: a cache-only engine other engines attach to
        if ((mi == 0 && mk == 0) || mi > (1u << 24)) return CUDIL_ERR_INVALID;
        CUDIL_CK(cudaGetDevice(&device));
        CUDIL_CK(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device));
        int rc = (threads == 128) ? configure<128>() : (threads == 256 ? configure<256>() : CUDIL_ERR_INVALID);
        if (rc) return rc;
        rc = configure_async();
        if (rc) return rc;
        rc = configure_wide();
        if (rc) return rc;
        prehash_grid = (int)std::min<size_t>((mi + kPrehashBlock - 1) / kPrehashBlock, (size_t)sm_count * 32);
        device_bytes = required_bytes(mk, mi);
        if (budget && device_bytes > budget) return CUDIL_ERR_BUDGET;
        sk_pitch = align256(C::SK_ROW);
        pk_pitch = align256(C::PK_ROW);
        scratch_bytes = scratch_for(mi);
        spec_slots = (unsigned)threads;
        // large batches (about 224 items per SM and more) default to the wide phased signer
        large_min_items = (size_t)224 * (size_t)sm_count;
        large_kernel = kWideVariant;
        large_spec = std::min<unsigned>(128u, 2u * (unsigned)threads);
        if ((mk && (cudaMalloc(&sk_cache, mk * sk_pitch) != cudaSuccess || cudaMalloc(&pk_cache, mk * pk_pitch) != cudaSuccess)) ||
            (mi && (cudaMalloc(&items, mi * C::ITEM_BYTES) != cudaSuccess || cudaMalloc(&best, mi * sizeof(unsigned)) != cudaSuccess ||
                    cudaMalloc(&locks, mi * sizeof(unsigned)) != cudaSuccess ||
                    cudaMalloc(&next_nonce, mi * sizeof(unsigned)) != cudaSuccess ||
                    cudaMalloc(&inflight, mi * sizeof(unsigned)) != cudaSuccess ||
                    cudaMalloc(&d_key, mi * sizeof(unsigned)) != cudaSuccess ||
                    cudaMalloc(&d_mlen, mi * sizeof(unsigned)) != cudaSuccess ||
                    cudaMalloc(&d_order, mi * sizeof(unsigned)) != cudaSuccess ||
                    cudaMalloc(&d_off, mi * sizeof(unsigned long long)) != cudaSuccess ||
                    cudaMalloc(&scratch, scratch_bytes) != cudaSuccess)) ||
            cudaMalloc(&q, sizeof(FusedQueue)) != cudaSuccess || cudaMallocHost(&h_stage, stage_bytes(mi)) != cudaSuccess ||
            cudaMallocHost(&h_status, sizeof(FusedQueue)) != cudaSuccess)
            return ::cudil::cudil_record_cuda_error(cudaGetLastError(), __FILE__, __LINE__);
        std::memset(h_status, 0, sizeof(FusedQueue));
        CUDIL_CK(cudaEventCreateWithFlags(&stage_ev, cudaEventDisableTiming));
        CUDIL_CK(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming));
        CUDIL_CK(cudaEventCreateWithFlags(&join_ev, cudaEventDisableTiming));
        CUDIL_CK(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
        CUDIL_CK(cudaMemset(q, 0, sizeof(FusedQueue)));
        return CUDIL_OK;
    }

    ~EngineImpl() override {
        if (g_sign) cudaGraphExecDestroy(g_sign);
        if (g_sign_large) cudaGraphExecDestroy(g_sign_large);
        if (g_verify) cudaGraphExecDestroy(g_verify);
        if (owns_cache) {
            cudaFree(sk_cache);
            cudaFree(pk_cache);
        }
        cudaFree(items);
        cudaFree(best);
        cudaFree(locks);
        cudaFree(next_nonce);
        cudaFree(inflight);
        cudaFree(q);
        cudaFree(d_key);
        cudaFree(d_mlen);
        cudaFree(d_order);
        cudaFree(d_off);
        cudaFree(scratch);
        if (h_stage) cudaFreeHost(h_stage);
        if (h_status) cudaFreeHost(h_status);
        if (stage_ev) cudaEventDestroy(stage_ev);
        if (fork_ev) cudaEventDestroy(fork_ev);
        if (join_ev) cudaEventDestroy(join_ev);
        if (side) cudaStreamDestroy(side);
    }

    // ------------------------------------------------------------ key caches
    // Use another engine's key caches (same parameter set); its caches must outlive this engine.
    int attach_keys(const EngineBase *src) {
        if (!src || src->mode != MODE || src == this) return CUDIL_ERR_INVALID;
        if (owns_cache) {
            cudaFree(sk_cache);
            cudaFree(pk_cache);
        }
        owns_cache = false;
        key_src = src->key_src ? src->key_src : src;  // the engine that owns the caches
        sk_cache = src->sk_cache;
        pk_cache = src->pk_cache;
        n_sk = src->n_sk;
        n_pk = src->n_pk;
        max_keys = src->max_keys;
        g_sign_key[0] = nullptr;  // re-capture graphs with the new cache pointers
        g_sign_large_key[0] = nullptr;
        g_verify_key[0] = nullptr;
        return CUDIL_OK;
    }

    int set_secret_keys(const uint8_t *d_sk, size_t nkeys, cudaStream_t st) {
        if (!d_sk || nkeys == 0 || nkeys > max_keys || !owns_cache) return CUDIL_ERR_INVALID;
        const int rc = build_sk_rows(d_sk, 0, nkeys, st);
        if (rc == CUDIL_OK) n_sk = nkeys;
        return rc;
    }

    // Cache rows [first, first + nkeys); first <= the number of rows built so far, so the built rows
    // stay one contiguous prefix.
    int update_secret_keys(const uint8_t *d_sk, size_t first, size_t nkeys, cudaStream_t st) {
        if (!d_sk || nkeys == 0 || first > n_sk || first > max_keys || nkeys > max_keys - first || !owns_cache)
            return CUDIL_ERR_INVALID;
        const int rc = build_sk_rows(d_sk, first, nkeys, st);
        if (rc == CUDIL_OK) n_sk = std::max(n_sk, first + nkeys);
        return rc;
    }

    // The unpack / transform of s1, s2, t0 (side stream) and ExpandA (caller's stream, rho read from
    // the packed keys) are independent and run concurrently; the caller's stream waits for both.
    int build_sk_rows(const uint8_t *d_sk, size_t first, size_t nkeys, cudaStream_t st) {
        const int nn = (int)nkeys;
        uint8_t *rows = sk_cache + first * sk_pitch;
        CUDIL_CK(cudaEventRecord(fork_ev, st));
        CUDIL_CK(cudaStreamWaitEvent(side, fork_ev, 0));
        CUDIL_LAUNCH(KID_CACHE_SK, side,
                     k_cache_sk<MODE><<<blocks_for(nkeys * (PM::L + 2 * PM::K + 1) * 16), kBlock, 0, side>>>(d_sk, rows, sk_pitch, nn));
        CUDIL_CK_LAUNCH();
        CUDIL_LAUNCH(KID_EXPAND_A, st,
                     k_expand_a_keys<MODE><<<blocks_for(nkeys * PM::K * PM::L), kBlock, 0, st>>>(d_sk, PM::SK_BYTES, rows, sk_pitch,
                                                                                             C::SK_MAT, nn));
        CUDIL_CK_LAUNCH();
        CUDIL_CK(cudaEventRecord(join_ev, side));
        CUDIL_CK(cudaStreamWaitEvent(st, join_ev, 0));
        return CUDIL_OK;
    }

    int set_public_keys(const uint8_t *d_pk, size_t nkeys, cudaStream_t st) {
        if (!d_pk || nkeys == 0 || nkeys > max_keys || !owns_cache) return CUDIL_ERR_INVALID;
        const int nn = (int)nkeys;
        // tr = H(pk) and t1_hat (side stream) run concurrently with ExpandA (rho from the packed keys)
        CUDIL_CK(cudaEventRecord(fork_ev, st));
        CUDIL_CK(cudaStreamWaitEvent(side, fork_ev, 0));
        CUDIL_LAUNCH(KID_CACHE_PK, side, k_cache_pk_tr<MODE><<<blocks_for(nkeys), kBlock, 0, side>>>(d_pk, pk_cache, pk_pitch, nn));
        CUDIL_CK_LAUNCH();
        CUDIL_LAUNCH(KID_CACHE_PK, side,
                     k_cache_pk_t1<MODE><<<blocks_for(nkeys * PM::K * 16), kBlock, 0, side>>>(d_pk, pk_cache, pk_pitch, nn));
        CUDIL_CK_LAUNCH();
        CUDIL_LAUNCH(KID_EXPAND_A, st,
                     k_expand_a_keys<MODE><<<blocks_for(nkeys * PM::K * PM::L), kBlock, 0, st>>>(d_pk, PM::PK_BYTES, pk_cache, pk_pitch,
                                                                                             C::PK_MAT, nn));
        CUDIL_CK_LAUNCH();
        CUDIL_CK(cudaEventRecord(join_ev, side));
        CUDIL_CK(cudaStreamWaitEvent(st, join_ev, 0));
        n_pk = nkeys;
        return CUDIL_OK;
    }

    // ------------------------------------------------------------ metadata upload
    int upload_meta(const unsigned long long *off, const unsigned *mlen, const unsigned *key, size_t n, size_t nkeys,
                    size_t msgs_bytes, bool longest_first, cudaStream_t st, const uint8_t *rho_seed = nullptr,
                    unsigned long long rho_counter = 0) {
        // the previous batch's copies out of the staging buffer must have completed (only those:
        // work the caller queued on the stream, such as input copies or cache builds, keeps
        // running while this batch is prepared)
        if (stage_pending) CUDIL_CK(cudaEventSynchronize(stage_ev));
        FusedQueue *hq = reinterpret_cast<FusedQueue *>(h_stage);
        std::memset(hq, 0, sizeof(FusedQueue));
        hq->n = (unsigned)n;
        if (rho_seed) {
            hq->rho_seeded = 1u;
            hq->rho_counter = rho_counter;
            std::memcpy(hq->rho_seed, rho_seed, sizeof hq->rho_seed);
        }
        unsigned *hk = reinterpret_cast<unsigned *>(h_stage + kStageHead);
        unsigned *hm = hk + max_items;
        unsigned *ho = hm + max_items;
        unsigned long long *hoff = reinterpret_cast<unsigned long long *>(ho + max_items);
        bool descending = true;  // already longest first (every batch of equal lengths is)
        for (size_t i = 0; i < n; ++i) {
            if (key[i] >= nkeys || (off[i] & 7u) || off[i] > msgs_bytes || mlen[i] > msgs_bytes - off[i])
                return CUDIL_ERR_INVALID;
            hk[i] = key[i];
            hm[i] = mlen[i];
            hoff[i] = off[i];
            if (i && mlen[i] > mlen[i - 1]) descending = false;
        }
        std::iota(ho, ho + n, 0u);
        if (longest_first && !descending)
            std::stable_sort(ho, ho + n, [&](unsigned a, unsigned b) { return hm[a] > hm[b]; });
        CUDIL_CK(cudaMemcpyAsync(q, hq, sizeof(FusedQueue), cudaMemcpyHostToDevice, st));
        CUDIL_CK(cudaMemcpyAsync(d_key, hk, n * sizeof(unsigned), cudaMemcpyHostToDevice, st));
        CUDIL_CK(cudaMemcpyAsync(d_mlen, hm, n * sizeof(unsigned), cudaMemcpyHostToDevice, st));
        CUDIL_CK(cudaMemcpyAsync(d_order, ho, n * sizeof(unsigned), cudaMemcpyHostToDevice, st));
        CUDIL_CK(cudaMemcpyAsync(d_off, hoff, n * sizeof(unsigned long long), cudaMemcpyHostToDevice, st));
        CUDIL_CK(cudaEventRecord(stage_ev, st));
        stage_pending = true;
        return CUDIL_OK;
    }

    // ------------------------------------------------------------ graphs
    template <int T>
    void record_sign(cudaStream_t st, uint8_t *d_sig, const uint8_t *d_msgs, const uint8_t *d_rhop, int variant,
                     unsigned spec) {
        MsgRefs mr{d_msgs, d_off, d_mlen, d_key, d_order, d_rhop, (unsigned)max_keys};
        k_fused_init<<<std::max(1, sm_count * 2), 256, 0, st>>>(q, best, locks, next_nonce, inflight);
        k_fused_prehash<MODE><<<prehash_grid, kPrehashBlock, 0, st>>>(sk_cache, sk_pitch, mr, items, q);
        FusedSignArgs a{sk_cache, sk_pitch, d_key, items, d_sig, (size_t)PM::SIG_BYTES, scratch, q, best, locks, next_nonce,
                        inflight, spec, nonce_limit, lock_spins, idle_polls, (unsigned)max_keys};
        if (variant == 1)
            k_fused_sign_async<MODE, 256, 64><<<async_grid[0], 256, async_smem[0], st>>>(a);
        else if (variant == 2)
            k_fused_sign_async<MODE, 512, 128><<<async_grid[1], 512, async_smem[1], st>>>(a);
        else if (variant == 3)
            k_fused_sign_async<MODE, 640, 160><<<async_grid[2], 640, async_smem[2], st>>>(a);
        else if (variant == 4)
            k_fused_sign_async<MODE, 768, 192><<<async_grid[3], 768, async_smem[3], st>>>(a);
        else if (variant == kWideVariant)
            k_fused_sign<MODE, kWideThreads><<<wide_grid, kWideThreads, wide_smem, st>>>(a);
        else
            k_fused_sign<MODE, T><<<sign_grid, T, sign_smem, st>>>(a);
        cudaMemcpyAsync(h_status, q, sizeof(FusedQueue), cudaMemcpyDeviceToHost, st);
    }

    template <int T>
    void record_verify(cudaStream_t st, int *d_ret, const uint8_t *d_sig, const uint8_t *d_msgs) {
        MsgRefs mr{d_msgs, d_off, d_mlen, d_key, d_order, nullptr, (unsigned)max_keys};
        k_fused_init<<<1, 32, 0, st>>>(q, nullptr, nullptr, nullptr, nullptr);
        k_fused_verify_prehash<MODE><<<prehash_grid, kPrehashBlock, 0, st>>>(pk_cache, pk_pitch, mr, items, q);
        k_fused_verify<MODE, T><<<verify_grid, T, verify_smem, st>>>(pk_cache, pk_pitch, mr, d_sig, PM::SIG_BYTES, d_ret,
                                                                    scratch, items, q);
        cudaMemcpyAsync(h_status, q, sizeof(FusedQueue), cudaMemcpyDeviceToHost, st);
    }

    int capture(cudaStream_t st, cudaGraphExec_t *exec, bool sign, uint8_t *out, const uint8_t *sig, const uint8_t *msgs,
                int variant = 0, unsigned spec = 0) {
        // graphs are captured on a private stream and launched on the caller's stream
        cudaStream_t cs;
        CUDIL_CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t graph;
        cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            if (sign)
                (threads == 128) ? record_sign<128>(cs, out, msgs, sig, variant, spec)
                                 : record_sign<256>(cs, out, msgs, sig, variant, spec);
            else
                (threads == 128) ? record_verify<128>(cs, reinterpret_cast<int *>(out), sig, msgs)
                                 : record_verify<256>(cs, reinterpret_cast<int *>(out), sig, msgs);
            e = cudaStreamEndCapture(cs, &graph);
        }
        cudaStreamDestroy(cs);
        (void)st;
        if (e != cudaSuccess) return cudil_record_cuda_error(e, __FILE__, __LINE__);
        if (*exec) cudaGraphExecDestroy(*exec);
        e = cudaGraphInstantiate(exec, graph, 0);
        cudaGraphDestroy(graph);
        return e == cudaSuccess ? CUDIL_OK : cudil_record_cuda_error(e, __FILE__, __LINE__);
    }

    // d_rhop: randomized signing seeds, 64 bytes per item (dense, device); nullptr = deterministic
    // rho_seed (host, 32 bytes): seeded randomized signing, rho' of item i derived on the device from
    // (rho_seed, rho_counter + i); it goes up with the batch metadata, so the graph is unchanged
    int sign(uint8_t *d_sig, const uint8_t *d_msgs, size_t msgs_bytes, const unsigned long long *off, const unsigned *mlen,
             const unsigned *key, size_t n, cudaStream_t st, const uint8_t *d_rhop = nullptr,
             const uint8_t *rho_seed = nullptr, unsigned long long rho_counter = 0) {
        if (n == 0) return CUDIL_OK;
        if (key_src) n_sk = key_src->n_sk;  // rows the owning engine has built by now
        if (!d_sig || !off || !mlen || !key || n > max_items || n_sk == 0) return CUDIL_ERR_INVALID;
        if (!d_msgs) {
            for (size_t i = 0; i < n; ++i)
                if (mlen[i]) return CUDIL_ERR_INVALID;
            d_msgs = reinterpret_cast<const uint8_t *>(items);  // any aligned pointer; never read
        }
        if (((uintptr_t)d_msgs) & 7u) return CUDIL_ERR_INVALID;
        const bool large = large_min_items && n >= large_min_items;
        cudaGraphExec_t &graph = large ? g_sign_large : g_sign;
        const void **gkey = large ? g_sign_large_key : g_sign_key;
        const bool recapture = !graph || gkey[0] != d_sig || gkey[1] != d_msgs || gkey[2] != d_rhop;
        // The signature rows may be device memory or pinned host memory (written by the signer over
        // PCIe as each signature is found); pageable host memory is refused before anything is queued.
        uint8_t *out = d_sig;
        if (recapture) {
            cudaPointerAttributes pa{};
            if (cudaPointerGetAttributes(&pa, d_sig) != cudaSuccess) {
                cudaGetLastError();
                return CUDIL_ERR_INVALID;
            }
            if (pa.type == cudaMemoryTypeUnregistered) return CUDIL_ERR_INVALID;
            if (pa.type == cudaMemoryTypeHost) {
                if (!pa.devicePointer) return CUDIL_ERR_INVALID;
                out = static_cast<uint8_t *>(pa.devicePointer);
            }
        }
        int rc = upload_meta(off, mlen, key, n, n_sk, msgs_bytes, true, st, rho_seed, rho_counter);
        if (rc) return rc;
        if (recapture) {
            // for a signing graph the `sig` argument of capture carries the randomized-signing seeds
            rc = capture(st, &graph, true, out, d_rhop, d_msgs, large ? large_kernel : sign_kernel,
                         large ? large_spec : spec_slots);
            if (rc) return rc;
            gkey[0] = d_sig;
            gkey[1] = d_msgs;
            gkey[2] = d_rhop;
        }
        CUDIL_LAUNCH(KID_FUSED_SIGN, st, cudaGraphLaunch(graph, st));
        CUDIL_CK_LAUNCH();
        Profiler::get().launches.fetch_add(2);  // the graph holds init + prehash + sign kernels
        last_n = n;
        return CUDIL_OK;
    }

    // Winning nonce per item of the last signing batch (kNonceExhausted: no accepted nonce below the
    // limit), copied into out (host or device memory) on st; returns after the copy completed.
    int last_nonces(unsigned *out, size_t n, cudaStream_t st) {
        if (!out || n > last_n || !best) return CUDIL_ERR_INVALID;
        if (n == 0) return CUDIL_OK;
        CUDIL_CK(cudaMemcpyAsync(out, best, n * sizeof(unsigned), cudaMemcpyDefault, st));
        CUDIL_CK(cudaStreamSynchronize(st));
        return CUDIL_OK;
    }

    // Bounds of the signer's loops; the signing graphs are re-captured on the next batch.
    int set_limits(unsigned nonces, unsigned spins, unsigned polls) {
        if (nonces == 0 || nonces > kNonceLimit) return CUDIL_ERR_INVALID;
        nonce_limit = nonces;
        lock_spins = spins;
        idle_polls = polls;
        g_sign_key[0] = nullptr;
        g_sign_large_key[0] = nullptr;
        return CUDIL_OK;
    }

    int verify(int *d_ret, const uint8_t *d_sig, const uint8_t *d_msgs, size_t msgs_bytes, const unsigned long long *off,
               const unsigned *mlen, const unsigned *key, size_t n, cudaStream_t st) {
        if (n == 0) return CUDIL_OK;
        if (key_src) n_pk = key_src->n_pk;
        if (!d_ret || !d_sig || !off || !mlen || !key || n > max_items || n_pk == 0) return CUDIL_ERR_INVALID;
        if (!d_msgs) {
            for (size_t i = 0; i < n; ++i)
                if (mlen[i]) return CUDIL_ERR_INVALID;
            d_msgs = reinterpret_cast<const uint8_t *>(items);
        }
        if (((uintptr_t)d_msgs) & 7u) return CUDIL_ERR_INVALID;
        int rc = upload_meta(off, mlen, key, n, n_pk, msgs_bytes, true, st);
        if (rc) return rc;
        if (!g_verify || g_verify_key[0] != d_ret || g_verify_key[1] != d_sig || d_msgs != g_verify_msgs) {
            rc = capture(st, &g_verify, false, reinterpret_cast<uint8_t *>(d_ret), d_sig, d_msgs);
            if (rc) return rc;
            g_verify_key[0] = d_ret;
            g_verify_key[1] = d_sig;
            g_verify_msgs = d_msgs;
        }
        CUDIL_LAUNCH(KID_FUSED_VERIFY, st, cudaGraphLaunch(g_verify, st));
        CUDIL_CK_LAUNCH();
        Profiler::get().launches.fetch_add(1);  // the graph holds init + verify kernels
        return CUDIL_OK;
    }

    const uint8_t *g_verify_msgs = nullptr;

    // Target of signing attempts in flight; the graph is re-captured on the next batch.
    int set_sign_kernel(int v) {
        if (v < 0 || v > kWideVariant) return CUDIL_ERR_INVALID;
        sign_kernel = v;
        g_sign_key[0] = nullptr;
        return CUDIL_OK;
    }

    int set_spec_slots(unsigned v) {
        spec_slots = v ? std::min<unsigned>(v, 2u * (unsigned)threads) : (unsigned)threads;
        g_sign_key[0] = nullptr;
        return CUDIL_OK;
    }

    int set_large_batch(size_t min_items, int variant, unsigned spec) {
        if (variant < 0 || variant > kWideVariant) return CUDIL_ERR_INVALID;
        large_min_items = min_items;
        large_kernel = variant;
        large_spec = spec ? std::min<unsigned>(spec, 2u * (unsigned)threads) : (unsigned)threads;
        g_sign_large_key[0] = nullptr;
        return CUDIL_OK;
    }
};

}  // namespace cudil
