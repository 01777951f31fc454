// Host orchestration of the plain (stage-by-stage) batched path, one instantiation per parameter
// set.  Mirrors the reference's host API (src/api.cu:26-515): caller-allocated pitched pools,
// asynchronous keypair/verify, and a sign scheduler that fills a task LUT with (item, nonce)
// attempts, speculating several consecutive nonces per item when fewer items than exec slots
// remain, and keeps for each item the accepted attempt of smallest nonce.
#pragma once

#include <climits>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/cudilithium.h"
#include "keypair_kernels.cuh"
#include "profiling.cuh"
#include "verify_kernels.cuh"

namespace cudil {

// Records the failing CUDA call of this host thread (cudil_last_error) and returns its status.
int cudil_record_cuda_error(cudaError_t e, const char *file, int line);
#define CUDIL_CK(x)                                                         \
    do {                                                                    \
        const cudaError_t cudil_e_ = (x);                                   \
        if (cudil_e_ != cudaSuccess) return ::cudil::cudil_record_cuda_error(cudil_e_, __FILE__, __LINE__); \
    } while (0)
#define CUDIL_CK_LAUNCH()                                                   \
    do {                                                                    \
        const cudaError_t cudil_e_ = cudaPeekAtLastError();                 \
        if (cudil_e_ != cudaSuccess) {                                      \
            (void)cudaGetLastError();                                       \
            return ::cudil::cudil_record_cuda_error(cudil_e_, __FILE__, __LINE__);   \
        }                                                                   \
    } while (0)

// Pools are addressed with 8- and 16-byte vector accesses: base and pitch must be 16-byte aligned
// (cudaMallocPitch pitches always are).
inline bool misaligned(const void *p, size_t pitch) { return ((uintptr_t)p & 15u) || (pitch & 15u); }

inline unsigned blocks_for(size_t threads, int per_block = kBlock) {
    return (unsigned)((threads + per_block - 1) / per_block);
}

__global__ void k_ntt_mul(const int32_t *a, const int32_t *b, int32_t *out, long long npolys);

template <int MODE>
struct Impl {
    using PM = P<MODE>;
    using LY = Layout<MODE>;
    static constexpr int K = PM::K, L = PM::L;
    // keys per keypair block, attempts per compute_w block, signatures per verify_w block:
    // chosen so that the 8 groups of a block have whole units of work in every phase.
    static constexpr int KPI = MODE == 2 ? 8 : (MODE == 3 ? 4 : 2);
    static constexpr int AW = MODE == 2 ? 2 : (MODE == 3 ? 4 : 1);
    static constexpr int AV = MODE == 2 ? 2 : (MODE == 3 ? 4 : 1);

    // ---------------------------------------------------------------- keypair
    static int keypair(uint8_t *pk, uint8_t *sk, const uint8_t *seeds, uint8_t *pool, size_t pitch, size_t n,
                       cudaStream_t st, size_t rand_index, cudaMemcpyKind in_kind, cudaMemcpyKind out_kind) {
        if (n == 0) return CUDIL_OK;
        if (!pk || !sk || !pool || pitch < LY::ref_keypair_row() || misaligned(pool, pitch) || n > (size_t)INT_MAX / 64)
            return CUDIL_ERR_INVALID;
        const int nn = (int)n;
        CUDIL_CK(cudaMemset2DAsync(pool + LY::KP_TACC, pitch, 0, (size_t)K * LY::POLY, n, st));
        if (seeds) CUDIL_CK(cudaMemcpy2DAsync(pool + LY::KP_SK + PM::SK_TR, pitch, seeds, SEEDBYTES, SEEDBYTES, n, in_kind, st));
        CUDIL_LAUNCH(KID_KP_SEED, st, k_kp_seed<MODE><<<blocks_for(n, kItemBlock), kItemBlock, 0, st>>>(pool, pitch, nn, (unsigned long long)rand_index, seeds ? 1 : 0));
        CUDIL_CK_LAUNCH();
        const size_t smem = KpSmem<MODE>::bytes(KPI);
        CUDIL_CK(cudaFuncSetAttribute(k_kp_main<MODE, KPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        CUDIL_LAUNCH(KID_KP_MAIN, st, k_kp_main<MODE, KPI><<<(unsigned)((n + KPI - 1) / KPI), kBlock, smem, st>>>(pool, pitch, nn));
        CUDIL_CK_LAUNCH();
        CUDIL_LAUNCH(KID_KP_TR, st, k_kp_tr<MODE><<<blocks_for(n, kItemBlock), kItemBlock, 0, st>>>(pool, pitch, nn));
        CUDIL_CK_LAUNCH();
        CUDIL_CK(cudaMemcpy2DAsync(pk, PM::PK_BYTES, pool + LY::KP_PK, pitch, PM::PK_BYTES, n, out_kind, st));
        CUDIL_CK(cudaMemcpy2DAsync(sk, PM::SK_BYTES, pool + LY::KP_SK, pitch, PM::SK_BYTES, n, out_kind, st));
        return CUDIL_OK;
    }

    // ---------------------------------------------------------------- sign
    // rhop: optional caller-supplied rho' rows (64 bytes, rhop_pitch apart, memory kind in_kind) for
    // randomized signing; nullptr = deterministic rho' = SHAKE256(K || mu).
    static int sign_setup(const uint8_t *m, size_t m_pitch, size_t mlen, const uint32_t *mlens, const uint8_t *sk,
                          size_t sk_pitch, uint8_t *pool, size_t sp, size_t n, cudaStream_t st, cudaMemcpyKind in_kind,
                          const uint8_t *rhop = nullptr, size_t rhop_pitch = 0) {
        const int nn = (int)n;
        if (mlen) CUDIL_CK(cudaMemcpy2DAsync(pool + LY::SG_MSG, sp, m, m_pitch, mlen, n, in_kind, st));
        CUDIL_CK(cudaMemcpy2DAsync(pool + LY::SG_SK, sp, sk, sk_pitch, PM::SK_BYTES, n, in_kind, st));
        if (rhop) CUDIL_CK(cudaMemcpy2DAsync(pool + LY::SG_RHOP, sp, rhop, rhop_pitch, CRHBYTES, n, in_kind, st));
        CUDIL_LAUNCH(KID_SIGN_PREHASH, st, k_sign_prehash<MODE><<<blocks_for(n, kItemBlock), kItemBlock, 0, st>>>(pool, sp, mlen, mlens, nn, rhop ? 1 : 0));
        CUDIL_CK_LAUNCH();
        CUDIL_LAUNCH(KID_EXPAND_A, st, k_expand_a<MODE><<<blocks_for(n * K * L), kBlock, 0, st>>>(pool, sp, LY::SG_SK + PM::SK_RHO, LY::sg_mat(mlen), nn));
        CUDIL_CK_LAUNCH();
        CUDIL_LAUNCH(KID_SIGN_UNPACK_NTT, st, k_sign_unpack_ntt<MODE><<<blocks_for(n * (L + 2 * K) * 16), kBlock, 0, st>>>(pool, sp, mlen, nn));
        CUDIL_CK_LAUNCH();
        return CUDIL_OK;
    }

    // One rejection round over nexec exec slots (exec LUT already on the device).
    static int sign_round(uint8_t *pool, size_t sp, size_t mlen, uint8_t *tpool, size_t tp, const uint32_t *d_exec,
                          uint8_t *d_done, int nexec, int nitems, cudaStream_t st) {
        CUDIL_LAUNCH(KID_SIGN_EXPAND_MASK, st, k_sign_expand_mask<MODE><<<blocks_for((size_t)nexec * L), kBlock, 0, st>>>(pool, sp, tpool, tp, d_exec, nexec, nitems));
        CUDIL_CK_LAUNCH();
        CUDIL_LAUNCH(KID_SIGN_COMPUTE_W, st, k_sign_compute_w<MODE, AW><<<(unsigned)((nexec + AW - 1) / AW), kBlock, 0, st>>>(pool, sp, mlen, tpool, tp, d_exec, nexec, nitems));
        CUDIL_CK_LAUNCH();
        CUDIL_LAUNCH(KID_SIGN_CHALLENGE, st, k_sign_challenge<MODE><<<blocks_for((size_t)nexec, kItemBlock), kItemBlock, 0, st>>>(pool, sp, tpool, tp, d_exec, nexec, nitems));
        CUDIL_CK_LAUNCH();
        CUDIL_LAUNCH(KID_SIGN_REJECT, st, k_sign_reject<MODE><<<blocks_for((size_t)nexec * 32), kBlock, 0, st>>>(pool, sp, mlen, tpool, tp, d_exec, d_done, nexec, nitems));
        CUDIL_CK_LAUNCH();
        return CUDIL_OK;
    }

    // mlens: optional device array of per-item message lengths (each <= mlen; rows of m hold the
    // message in their first mlens[i] bytes); nullptr = every message is mlen bytes.
    static int sign(uint8_t *sig, size_t sig_pitch, size_t *siglen, const uint8_t *m, size_t m_pitch, size_t mlen,
                    const uint8_t *sk, size_t sk_pitch, uint8_t *pool, size_t sp, uint8_t *tpool, size_t tp,
                    cudil_task_lut *lut, size_t T, size_t n, cudaStream_t st, cudaMemcpyKind in_kind,
                    cudaMemcpyKind out_kind, const uint32_t *mlens = nullptr, const uint8_t *rhop = nullptr,
                    size_t rhop_pitch = 0) {
        if (siglen) *siglen = PM::SIG_BYTES;
        if (n == 0) return CUDIL_OK;
        if (!sig || !sk || (!m && mlen) || !pool || !tpool || !lut || T == 0 || n > 65536) return CUDIL_ERR_INVALID;
        if (sp < LY::ref_sign_row(mlen) || tp < LY::ref_sign_temp_row() || sig_pitch < (size_t)PM::SIG_BYTES ||
            (mlen && m_pitch < mlen) || T > (size_t)INT_MAX / 64 || misaligned(pool, sp) || misaligned(tpool, tp))
            return CUDIL_ERR_INVALID;
        if (!lut->sign_lut || lut->sign_lut_len != n || !lut->h_exec_lut || !lut->h_done_lut || !lut->h_copy_lut ||
            !lut->d_exec_lut || !lut->d_done_lut || !lut->d_copy_lut)
            return CUDIL_ERR_INVALID;
        if (rhop && rhop_pitch < (size_t)CRHBYTES) return CUDIL_ERR_INVALID;
        int rc = sign_setup(m, m_pitch, mlen, mlens, sk, sk_pitch, pool, sp, n, st, in_kind, rhop, rhop_pitch);
        if (rc) return rc;

        cudil_sign_lut_element *sl = lut->sign_lut;
        for (size_t i = 0; i < n; ++i) {
            sl[i].done_flag = 0;
            sl[i].nonce = 0;
        }
        size_t remaining = n;
        size_t rounds = 0;
        std::vector<uint32_t> pending;
        pending.reserve(n);
        while (remaining) {
            if (++rounds > (size_t)1 << 20) return CUDIL_ERR_TIMEOUT;
            // fill every exec slot, cycling over pending items in index order with consecutive
            // nonces (the exec order of src/api.cu:221-232 and :322-332); the pending list keeps
            // the fill linear in T when few items remain
            pending.clear();
            for (size_t s = 0; s < n; ++s)
                if (!sl[s].done_flag) pending.push_back((uint32_t)s);
            size_t e = 0;
            while (e < T) {
                for (size_t q = 0; q < pending.size() && e < T; ++q) {
                    const uint32_t s = pending[q];
                    lut->h_exec_lut[e++] = (s << 16) | (uint32_t)(sl[s].nonce++);
                }
            }
            CUDIL_CK(cudaMemcpyAsync(lut->d_exec_lut, lut->h_exec_lut, sizeof(uint32_t) * T, cudaMemcpyHostToDevice, st));
            CUDIL_CK(cudaMemsetAsync(lut->d_done_lut, 0, T, st));
            rc = sign_round(pool, sp, mlen, tpool, tp, lut->d_exec_lut, lut->d_done_lut, (int)T, (int)n, st);
            if (rc) return rc;
            CUDIL_CK(cudaMemcpyAsync(lut->h_done_lut, lut->d_done_lut, T, cudaMemcpyDeviceToHost, st));
            CUDIL_CK(cudaStreamSynchronize(st));
            // first accepted slot of an item in exec order = its smallest accepted nonce
            size_t cc = 0;
            for (size_t x = 0; x < T; ++x) {
                if (!lut->h_done_lut[x]) continue;
                const size_t s = lut->h_exec_lut[x] >> 16;
                if (sl[s].done_flag) continue;
                sl[s].done_flag = 1;
                lut->h_copy_lut[cc].exec_idx = x;
                lut->h_copy_lut[cc].sign_idx = s;
                ++cc;
                --remaining;
            }
            if (cc) {
                CUDIL_CK(cudaMemcpyAsync(lut->d_copy_lut, lut->h_copy_lut, sizeof(cudil_copy_lut_element) * cc,
                                         cudaMemcpyHostToDevice, st));
                CUDIL_LAUNCH(KID_SIG_COPY, st, k_sig_copy<MODE><<<(unsigned)cc, 128, 0, st>>>(pool, sp, tpool, tp,
                                                               reinterpret_cast<const CopyEntry *>(lut->d_copy_lut), T, n));
                CUDIL_CK_LAUNCH();
            }
        }
        CUDIL_CK(cudaMemcpy2DAsync(sig, sig_pitch, pool + LY::SG_SIG, sp, PM::SIG_BYTES, n, out_kind, st));
        return CUDIL_OK;
    }

    // ---------------------------------------------------------------- verify
    static int verify(int *ret, const uint8_t *sig, size_t sig_pitch, size_t siglen, const uint8_t *m, size_t m_pitch,
                      size_t mlen, const uint8_t *pk, size_t pk_pitch, uint8_t *pool, size_t pitch, size_t n,
                      cudaStream_t st, cudaMemcpyKind in_kind, cudaMemcpyKind out_kind, const uint32_t *mlens = nullptr) {
        if (n == 0) return CUDIL_OK;
        if (!ret) return CUDIL_ERR_INVALID;
        if (siglen != (size_t)PM::SIG_BYTES) {
            if (out_kind == cudaMemcpyDeviceToHost) {
                for (size_t i = 0; i < n; ++i) ret[i] = -1;
            } else {
                CUDIL_CK(cudaMemsetAsync(ret, 0xFF, n * sizeof(int), st));
            }
            return CUDIL_OK;
        }
        if (!sig || !pk || (!m && mlen) || !pool || pitch < LY::ref_verify_row(mlen) || sig_pitch < (size_t)PM::SIG_BYTES ||
            (mlen && m_pitch < mlen) || n > (size_t)INT_MAX / 64 || misaligned(pool, pitch))
            return CUDIL_ERR_INVALID;
        const int nn = (int)n;
        CUDIL_CK(cudaMemcpy2DAsync(pool + LY::VF_SIG, pitch, sig, sig_pitch, PM::SIG_BYTES, n, in_kind, st));
        if (mlen) CUDIL_CK(cudaMemcpy2DAsync(pool + LY::VF_TRM + SEEDBYTES, pitch, m, m_pitch, mlen, n, in_kind, st));
        CUDIL_CK(cudaMemcpy2DAsync(pool + LY::VF_PK, pitch, pk, pk_pitch, PM::PK_BYTES, n, in_kind, st));
        CUDIL_LAUNCH(KID_VERIFY_PREPARE, st, k_verify_prepare<MODE><<<blocks_for(n, kItemBlock), kItemBlock, 0, st>>>(pool, pitch, mlen, mlens, nn));
        CUDIL_CK_LAUNCH();
        CUDIL_LAUNCH(KID_EXPAND_A, st, k_expand_a<MODE><<<blocks_for(n * K * L), kBlock, 0, st>>>(pool, pitch, LY::VF_PK, LY::vf_mat(mlen), nn));
        CUDIL_CK_LAUNCH();
        CUDIL_LAUNCH(KID_VERIFY_W, st, k_verify_w<MODE, AV><<<(unsigned)((n + AV - 1) / AV), kBlock, 0, st>>>(pool, pitch, mlen, nn));
        CUDIL_CK_LAUNCH();
        CUDIL_LAUNCH(KID_VERIFY_FINAL, st, k_verify_final<MODE><<<blocks_for(n, kItemBlock), kItemBlock, 0, st>>>(pool, pitch, mlen, nn));
        CUDIL_CK_LAUNCH();
        CUDIL_CK(cudaMemcpy2DAsync(ret, sizeof(int), pool + LY::vf_aux(mlen) + 68, pitch, sizeof(int), n, out_kind, st));
        return CUDIL_OK;
    }
};

}  // namespace cudil
