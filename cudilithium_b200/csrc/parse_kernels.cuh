// Batched well-formedness checks of encodings, run as a step of their own (for example by a
// server before it queues a request).  Status per item:
//   signatures (k_sig_check): bit 0 = hint encoding invalid -- per-polynomial end counts
//     non-decreasing and at most omega, positions strictly increasing inside a polynomial, unused
//     slots zero (src/verify.cu:51-93); bit 1 = some z coefficient with |z| >= gamma1 - beta (the
//     z check of src/verify.cu:98-121).  Verification rejects every signature with a bit set.
//   secret keys (k_sk_check): bit 0 = an s1 / s2 coefficient field outside [0, 2 eta] (the
//     eta - s encoding of src/keypair.cu:116-130).
// Public keys need no check: every byte string of the right length is a valid t1 encoding.
#pragma once

#include "sign_kernels.cuh"

namespace cudil {

// One warp per signature: lane 0 walks the hint section (omega + k bytes), all lanes test the z
// coefficients.
template <int MODE>
__global__ void __launch_bounds__(kBlock) k_sig_check(int *status, const uint8_t *sig, size_t sig_pitch, int n) {
    using PM = P<MODE>;
    constexpr int K = PM::K, L = PM::L, OMEGA = PM::OMEGA, ZB = PM::Z_BITS;
    const int it = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (it >= n) return;
    const uint8_t *s = sig + (size_t)it * sig_pitch;
    int st = 0;
    if (lane == 0) {
        const uint8_t *h = s + PM::SIG_H;
        int k = 0;
        for (int i = 0; i < K && !st; ++i) {
            const int end = h[OMEGA + i];
            if (end < k || end > OMEGA) {
                st = 1;
                break;
            }
            for (int j = k + 1; j < end; ++j)
                if (h[j] <= h[j - 1]) st = 1;
            k = end;
        }
        if (!st)
            for (int j = k; j < OMEGA; ++j)
                if (h[j]) st = 1;
    }
    // z field c occupies bits [c * ZB, (c + 1) * ZB) of the z section; get_bits reads at most 4
    // bytes from the field's first byte, which stay inside the signature (the hints follow z)
    bool bad = false;
    for (int c = lane; c < L * N; c += 32) {
        const int32_t z = PM::GAMMA1 - (int32_t)get_bits(s + SEEDBYTES, c * ZB, ZB);
        bad |= exceeds(z, PM::GAMMA1 - PM::BETA);
    }
    if (__ballot_sync(0xFFFFFFFFu, bad)) st |= 2;
    if (lane == 0) status[it] = st;
}

// One warp per secret key: lanes test the eta fields of s1 and s2.
template <int MODE>
__global__ void __launch_bounds__(kBlock) k_sk_check(int *status, const uint8_t *sk, int n) {
    using PM = P<MODE>;
    constexpr int NP = PM::L + PM::K, EB = PM::ETA_BITS;
    const int it = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (it >= n) return;
    const uint8_t *s = sk + (size_t)it * PM::SK_BYTES + PM::SK_S1;
    bool bad = false;
    for (int c = lane; c < NP * N; c += 32) {
        const int poly = c / N, k = c % N;
        const uint8_t *p = s + (size_t)poly * PM::POLYETA_PACKED;
        const int bit = k * EB, byte = bit >> 3, sh = bit & 7;
        // a 3- or 4-bit field spans at most two bytes; the second is read only when needed
        uint32_t v = (uint32_t)p[byte] >> sh;
        if (sh + EB > 8) v |= (uint32_t)p[byte + 1] << (8 - sh);
        bad |= (int)(v & ((1u << EB) - 1u)) > 2 * PM::ETA;
    }
    const bool any = __ballot_sync(0xFFFFFFFFu, bad) != 0u;
    if (lane == 0) status[it] = any ? 1 : 0;
}

}  // namespace cudil
