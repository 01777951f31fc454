/*
 * Drop-in replacement for the reference's per-mode C++ API (include/api.cuh:27-63 and the
 * parameter macros of include/params.h), implemented inline on the C ABI of cudilithium.h.
 *
 * Like the reference, one translation unit serves one parameter set, chosen at compile time with
 * DILITHIUM_MODE (2, 3 or 5; default 2).  A program written against the reference's api.cuh
 * compiles unchanged against this header and links with libcudilithium_b200.so instead of the
 * reference's per-mode library:
 *
 *   reference                                  this header
 *   crypto_sign_keypair   (src/api.cu:26-61)   -> cudil_keypair
 *   crypto_sign_signature (src/api.cu:63-452)  -> cudil_sign
 *   crypto_sign_verify    (src/api.cu:454-515) -> cudil_verify
 *
 * Argument meaning, default arguments, pool pitches, the task_lut protocol (the caller resizes
 * sign_lut to batch_size and allocates the exec/done/copy arrays of exec_threshold entries) and
 * return values are the reference's: both functions return 0 and verify results go to ret[i]
 * (0 valid, -1 invalid).  Unlike the reference, an invalid argument (unsupported pitch or size,
 * missing buffer) or a CUDA failure is reported: crypto_sign_keypair / crypto_sign_signature
 * return the negative cudilithium status, crypto_sign_verify sets every ret[i] = -1.
 *
 * Defining DILITHIUM_RANDOMIZED_SIGNING (as for the reference) makes crypto_sign_signature draw the
 * 64-byte rho' of every message from /dev/urandom and sign with cudil_sign_randomized.  The
 * rho' buffer is pageable host memory, so the reference's asynchronous upload of it becomes a
 * synchronous copy; every other step is unchanged.
 *
 * The parameter macros keep the names of the Dilithium specification's reference code, which the
 * reference's params.h uses, so pool sizes computed from them are the reference's.
 */
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "cudilithium.h"

#ifndef DILITHIUM_MODE
#define DILITHIUM_MODE 2
#endif

#define SEEDBYTES 32
#define CRHBYTES 64
#define DILITHIUM_N 256
#define DILITHIUM_Q 8380417
#define DILITHIUM_D 13
#define POLYT1_PACKEDBYTES 320
#define POLYT0_PACKEDBYTES 416

#if DILITHIUM_MODE == 2
#define DILITHIUM_K 4
#define DILITHIUM_L 4
#define DILITHIUM_ETA 2
#define DILITHIUM_TAU 39
#define DILITHIUM_BETA 78
#define DILITHIUM_GAMMA1 (1 << 17)
#define DILITHIUM_GAMMA2 ((DILITHIUM_Q - 1) / 88)
#define DILITHIUM_OMEGA 80
#elif DILITHIUM_MODE == 3
#define DILITHIUM_K 6
#define DILITHIUM_L 5
#define DILITHIUM_ETA 4
#define DILITHIUM_TAU 49
#define DILITHIUM_BETA 196
#define DILITHIUM_GAMMA1 (1 << 19)
#define DILITHIUM_GAMMA2 ((DILITHIUM_Q - 1) / 32)
#define DILITHIUM_OMEGA 55
#elif DILITHIUM_MODE == 5
#define DILITHIUM_K 8
#define DILITHIUM_L 7
#define DILITHIUM_ETA 2
#define DILITHIUM_TAU 60
#define DILITHIUM_BETA 120
#define DILITHIUM_GAMMA1 (1 << 19)
#define DILITHIUM_GAMMA2 ((DILITHIUM_Q - 1) / 32)
#define DILITHIUM_OMEGA 75
#else
#error "DILITHIUM_MODE must be 2, 3 or 5"
#endif

#if DILITHIUM_GAMMA1 == (1 << 17)
#define POLYZ_PACKEDBYTES 576
#else
#define POLYZ_PACKEDBYTES 640
#endif
#if DILITHIUM_GAMMA2 == (DILITHIUM_Q - 1) / 88
#define POLYW1_PACKEDBYTES 192
#else
#define POLYW1_PACKEDBYTES 128
#endif
#if DILITHIUM_ETA == 2
#define POLYETA_PACKEDBYTES 96
#else
#define POLYETA_PACKEDBYTES 128
#endif
#define POLYVECH_PACKEDBYTES (DILITHIUM_OMEGA + DILITHIUM_K)

#define CRYPTO_PUBLICKEYBYTES (SEEDBYTES + DILITHIUM_K * POLYT1_PACKEDBYTES)
#define CRYPTO_SECRETKEYBYTES                                                                          \
    (3 * SEEDBYTES + DILITHIUM_L * POLYETA_PACKEDBYTES + DILITHIUM_K * POLYETA_PACKEDBYTES +           \
     DILITHIUM_K * POLYT0_PACKEDBYTES)
#define CRYPTO_BYTES (SEEDBYTES + DILITHIUM_L * POLYZ_PACKEDBYTES + POLYVECH_PACKEDBYTES)

#define ALIGN_TO_256_BYTES(x) ((((x) + 255) / 256) * 256)

struct sign_lut_element {
    int done_flag = 0;
    uint16_t nonce = 0;
};

struct copy_lut_element {
    size_t exec_idx;
    size_t sign_idx;
};

struct task_lut {
    std::vector<sign_lut_element> sign_lut;
    uint32_t *h_exec_lut;
    uint8_t *h_done_lut;
    copy_lut_element *h_copy_lut;
    uint32_t *d_exec_lut;
    uint8_t *d_done_lut;
    copy_lut_element *d_copy_lut;
};

static_assert(sizeof(sign_lut_element) == sizeof(cudil_sign_lut_element), "sign_lut_element layout");
static_assert(sizeof(copy_lut_element) == sizeof(cudil_copy_lut_element), "copy_lut_element layout");

inline int crypto_sign_keypair(uint8_t *pk, uint8_t *sk, uint8_t *d_keypair_mem_pool, size_t keypair_mem_pool_pitch,
                               size_t batch_size = 1, cudaStream_t stream = nullptr, size_t rand_index = 0) {
    return cudil_keypair(DILITHIUM_MODE, pk, sk, d_keypair_mem_pool, keypair_mem_pool_pitch, batch_size,
                         (void *)stream, rand_index);
}

#ifdef DILITHIUM_RANDOMIZED_SIGNING
// rho' from the operating system's random source, as the reference's randombytes (src/api.cu:143-148)
inline bool cudil_os_random(uint8_t *out, size_t n) {
    FILE *f = std::fopen("/dev/urandom", "rb");
    if (!f) return false;
    const bool ok = std::fread(out, 1, n, f) == n;
    std::fclose(f);
    return ok;
}
#endif

inline int crypto_sign_signature(uint8_t *sig, size_t sig_pitch, size_t *siglen, const uint8_t *m, size_t m_pitch,
                                 size_t mlen, const uint8_t *sk, uint8_t *d_sign_mem_pool,
                                 size_t d_sign_mem_pool_pitch, uint8_t *d_temp_mem_pool,
                                 size_t d_temp_mem_pool_pitch, task_lut &lut, size_t exec_threshold,
                                 size_t batch_size = 1, cudaStream_t stream = nullptr) {
    cudil_task_lut c{};
    c.sign_lut = reinterpret_cast<cudil_sign_lut_element *>(lut.sign_lut.data());
    c.sign_lut_len = lut.sign_lut.size();
    c.h_exec_lut = lut.h_exec_lut;
    c.h_done_lut = lut.h_done_lut;
    c.h_copy_lut = reinterpret_cast<cudil_copy_lut_element *>(lut.h_copy_lut);
    c.d_exec_lut = lut.d_exec_lut;
    c.d_done_lut = lut.d_done_lut;
    c.d_copy_lut = reinterpret_cast<cudil_copy_lut_element *>(lut.d_copy_lut);
#ifdef DILITHIUM_RANDOMIZED_SIGNING
    std::vector<uint8_t> rhoprime(batch_size * CRHBYTES);
    if (batch_size && !cudil_os_random(rhoprime.data(), rhoprime.size())) return CUDIL_ERR_INVALID;
    return cudil_sign_randomized(DILITHIUM_MODE, sig, sig_pitch, siglen, m, m_pitch, mlen, sk, rhoprime.data(), CRHBYTES,
                                 d_sign_mem_pool, d_sign_mem_pool_pitch, d_temp_mem_pool, d_temp_mem_pool_pitch, &c,
                                 exec_threshold, batch_size, (void *)stream);
#else
    return cudil_sign(DILITHIUM_MODE, sig, sig_pitch, siglen, m, m_pitch, mlen, sk, d_sign_mem_pool,
                      d_sign_mem_pool_pitch, d_temp_mem_pool, d_temp_mem_pool_pitch, &c, exec_threshold, batch_size,
                      (void *)stream);
#endif
}

inline void crypto_sign_verify(int *ret, const uint8_t *sig, size_t sig_pitch, size_t siglen, const uint8_t *m,
                               size_t m_pitch, size_t mlen, const uint8_t *pk, uint8_t *d_verify_mem_pool,
                               size_t verify_mem_pool_pitch, size_t batch_size = 1, cudaStream_t stream = nullptr) {
    const int rc = cudil_verify(DILITHIUM_MODE, ret, sig, sig_pitch, siglen, m, m_pitch, mlen, pk, d_verify_mem_pool,
                                verify_mem_pool_pitch, batch_size, (void *)stream);
    if (rc != CUDIL_OK && ret)
        for (size_t i = 0; i < batch_size; ++i) ret[i] = -1;
}
