// Launch accounting for the library's kernels: a process-wide launch counter (always on) and
// optional per-kernel CUDA-event timing on the launching stream (off by default; enabled with
// cudil_kernel_timing(1)).  Used by the benchmark to report how many kernels ran in a timed
// region and which kernel dominates it.
#pragma once

#include <atomic>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

namespace cudil {

enum KernelId : int {
    KID_KP_SEED = 0,
    KID_KP_MAIN,
    KID_KP_TR,
    KID_SIGN_PREHASH,
    KID_EXPAND_A,
    KID_SIGN_UNPACK_NTT,
    KID_SIGN_EXPAND_MASK,
    KID_SIGN_COMPUTE_W,
    KID_SIGN_CHALLENGE,
    KID_SIGN_REJECT,
    KID_SIG_COPY,
    KID_VERIFY_PREPARE,
    KID_VERIFY_W,
    KID_VERIFY_FINAL,
    KID_NTT_MUL,
    KID_ALU_PEAK,
    KID_FUSED_SIGN,
    KID_FUSED_VERIFY,
    KID_FUSED_SCHED,
    KID_CACHE_SK,
    KID_CACHE_PK,
    KID_SIG_CHECK,
    KID_SK_CHECK,
    KID_DERIVE_RHOP,
    KID_COUNT
};

inline const char *kernel_name(int id) {
    static const char *names[KID_COUNT] = {
        "k_kp_seed", "k_kp_main", "k_kp_tr", "k_sign_prehash", "k_expand_a", "k_sign_unpack_ntt",
        "k_sign_expand_mask", "k_sign_compute_w", "k_sign_challenge", "k_sign_reject", "k_sig_copy",
        "k_verify_prepare", "k_verify_w", "k_verify_final", "k_ntt_mul", "k_alu_peak",
        "k_fused_sign (graph)", "k_fused_verify (graph)", "k_fused_sched", "k_cache_sk", "k_cache_pk",
        "k_sig_check", "k_sk_check", "k_derive_rhoprime"};
    return (id >= 0 && id < KID_COUNT) ? names[id] : "?";
}

struct Profiler {
    std::atomic<unsigned long long> launches{0};
    std::atomic<int> timing{0};
    std::mutex mu;
    struct Pending {
        int id;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending;
    double total_ms[KID_COUNT] = {};
    unsigned long long count[KID_COUNT] = {};

    static Profiler &get() {
        static Profiler p;
        return p;
    }

    // Returns the start event to pass to after(), or nullptr when timing is off.
    cudaEvent_t before(cudaStream_t st) {
        launches.fetch_add(1, std::memory_order_relaxed);
        if (!timing.load(std::memory_order_relaxed)) return nullptr;
        cudaEvent_t a;
        if (cudaEventCreate(&a) != cudaSuccess) return nullptr;
        cudaEventRecord(a, st);
        return a;
    }

    void after(int id, cudaEvent_t a, cudaStream_t st) {
        if (!a) return;
        cudaEvent_t b;
        if (cudaEventCreate(&b) != cudaSuccess) {
            cudaEventDestroy(a);
            return;
        }
        cudaEventRecord(b, st);
        std::lock_guard<std::mutex> g(mu);
        pending.push_back({id, a, b});
    }

    void collect() {
        std::lock_guard<std::mutex> g(mu);
        for (auto &p : pending) {
            float ms = 0.f;
            cudaEventSynchronize(p.b);
            if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
                total_ms[p.id] += ms;
                count[p.id] += 1;
            }
            cudaEventDestroy(p.a);
            cudaEventDestroy(p.b);
        }
        pending.clear();
    }

    void reset() {
        collect();
        std::lock_guard<std::mutex> g(mu);
        for (int i = 0; i < KID_COUNT; ++i) {
            total_ms[i] = 0;
            count[i] = 0;
        }
    }
};

}  // namespace cudil

// Launch a kernel with accounting: CUDIL_LAUNCH(id, stream, kernel<<<grid, block, smem, stream>>>(args)).
#define CUDIL_LAUNCH(id, st, ...)                                       \
    do {                                                                \
        cudaEvent_t cudil_ev_ = ::cudil::Profiler::get().before(st);    \
        __VA_ARGS__;                                                    \
        ::cudil::Profiler::get().after((id), cudil_ev_, (st));          \
    } while (0)
