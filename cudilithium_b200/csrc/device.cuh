// Device routines shared by the keypair / sign / verify kernels: SHAKE-stream samplers run by one
// thread per stream, and 16-thread-group polynomial helpers.
#pragma once

#include <cstdint>

#include "arith.cuh"
#include "bounds.cuh"
#include "keccak.cuh"
#include "ntt.cuh"
#include "params.cuh"

namespace cudil {

__device__ __forceinline__ uint2 ld_lane(const uint8_t *p) { return *reinterpret_cast<const uint2 *>(p); }

template <int NL>
__device__ __forceinline__ void ld_lanes(uint2 (&v)[NL], const uint8_t *p) {
#pragma unroll
    for (int i = 0; i < NL; ++i) v[i] = ld_lane(p + 8 * i);
}

// ExpandA entry A[i][j] (NTT domain): SHAKE128(rho || j || i), 23-bit little-endian candidates
// accepted below q (src/sign.cu:98-163, src/keypair.cu:139-190; the stream is extended until 256
// coefficients are accepted, as benches/bench_rej_sampling.cu:571-593 does).  `emit(ctr, v)` is
// called for every accepted coefficient in order.
template <typename Emit>
__device__ __forceinline__ void expand_a_stream(const uint2 (&rho)[4], int i, int j, Emit emit) {
    uint32_t al[25], ah[25];
    shake_absorb_seed_nonce<SHAKE128_RATE, 4>(al, ah, rho, (uint32_t)((i << 8) | j));
    int ctr = 0;
#pragma unroll 1
    while (ctr < N) {
        keccak_f1600(al, ah);
        // 21 lanes = 7 groups of 3 lanes = 7 x 8 candidates of 3 bytes.
#pragma unroll
        for (int g = 0; g < 7; ++g) {
            const uint32_t w0 = al[3 * g], w1 = ah[3 * g], w2 = al[3 * g + 1];
            const uint32_t w3 = ah[3 * g + 1], w4 = al[3 * g + 2], w5 = ah[3 * g + 2];
            uint32_t c[8];
            c[0] = w0;
            c[1] = __funnelshift_r(w0, w1, 24);
            c[2] = __funnelshift_r(w1, w2, 16);
            c[3] = w2 >> 8;
            c[4] = w3;
            c[5] = __funnelshift_r(w3, w4, 24);
            c[6] = __funnelshift_r(w4, w5, 16);
            c[7] = w5 >> 8;
#pragma unroll
            for (int m = 0; m < 8; ++m) {
                const uint32_t v = c[m] & 0x7FFFFFu;
                if (v < (uint32_t)Q && ctr < N) {
                    emit(ctr, (int32_t)v);
                    ++ctr;
                }
            }
        }
    }
}

// The same entry written to out[0..255].  Where out is 16-byte aligned, a group of eight
// candidates that are all accepted while the count is a multiple of four goes out as two 16-byte
// stores; anything else is stored coefficient by coefficient (a candidate is rejected with
// probability (2^23 - q) / 2^23 < 0.1%, so nearly every group takes the wide path).
__device__ __forceinline__ void expand_a_row(const uint2 (&rho)[4], int i, int j, int32_t *out) {
    uint32_t al[25], ah[25];
    shake_absorb_seed_nonce<SHAKE128_RATE, 4>(al, ah, rho, (uint32_t)((i << 8) | j));
    const bool wide = (reinterpret_cast<uintptr_t>(out) & 15u) == 0u;
    int ctr = 0;
#pragma unroll 1
    while (ctr < N) {
        keccak_f1600(al, ah);
#pragma unroll
        for (int g = 0; g < 7; ++g) {
            const uint32_t w0 = al[3 * g], w1 = ah[3 * g], w2 = al[3 * g + 1];
            const uint32_t w3 = ah[3 * g + 1], w4 = al[3 * g + 2], w5 = ah[3 * g + 2];
            uint32_t c[8];
            c[0] = w0;
            c[1] = __funnelshift_r(w0, w1, 24);
            c[2] = __funnelshift_r(w1, w2, 16);
            c[3] = w2 >> 8;
            c[4] = w3;
            c[5] = __funnelshift_r(w3, w4, 24);
            c[6] = __funnelshift_r(w4, w5, 16);
            c[7] = w5 >> 8;
            bool all = true;
#pragma unroll
            for (int m = 0; m < 8; ++m) {
                c[m] &= 0x7FFFFFu;
                all &= c[m] < (uint32_t)Q;
            }
            if (wide && all && (ctr & 3) == 0 && ctr + 8 <= N) {
                int4 *o = reinterpret_cast<int4 *>(out + ctr);
                o[0] = make_int4((int)c[0], (int)c[1], (int)c[2], (int)c[3]);
                o[1] = make_int4((int)c[4], (int)c[5], (int)c[6], (int)c[7]);
                ctr += 8;
            } else {
#pragma unroll
                for (int m = 0; m < 8; ++m) {
                    if (c[m] < (uint32_t)Q && ctr < N) {
                        out[ctr] = (int32_t)c[m];
                        ++ctr;
                    }
                }
            }
        }
    }
}

// ExpandS entry: SHAKE256(rho' || nonce), nibbles < 15 (eta 2) or < 9 (eta 4), low nibble first
// (src/keypair.cu:84-114).  emit(ctr, s) with s in [-eta, eta].
template <int MODE, typename Emit>
__device__ __forceinline__ void expand_s_stream(const uint2 (&rhoprime)[8], int nonce, Emit emit) {
    constexpr int ETA = Params<MODE>::ETA;
    uint32_t al[25], ah[25];
    shake_absorb_seed_nonce<SHAKE256_RATE, 8>(al, ah, rhoprime, (uint32_t)nonce);
    int ctr = 0;
#pragma unroll 1
    while (ctr < N) {
        keccak_f1600(al, ah);
#pragma unroll
        for (int w = 0; w < 17; ++w) {
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                const uint32_t word = half ? ah[w] : al[w];
#pragma unroll
                for (int nb = 0; nb < 8; ++nb) {
                    const uint32_t t = (word >> (4 * nb)) & 15u;
                    if constexpr (ETA == 2) {
                        if (t < 15 && ctr < N) {
                            emit(ctr, 2 - (int32_t)(t - (205 * t >> 10) * 5));
                            ++ctr;
                        }
                    } else {
                        if (t < 9 && ctr < N) {
                            emit(ctr, 4 - (int32_t)t);
                            ++ctr;
                        }
                    }
                }
            }
        }
    }
}

// ExpandMask entry y_j: SHAKE256(rho' || kappa) with kappa = L*nonce + j (src/sign.cu:488-499);
// the first POLYZ_PACKED bytes are stored verbatim (gamma1 - y packing), `out` 8-byte aligned.
template <int MODE>
__device__ __forceinline__ void expand_mask_stream(uint8_t *out, const uint2 (&rhoprime)[8], uint32_t kappa) {
    constexpr int LANES = P<MODE>::POLYZ_PACKED / 8;  // 72 or 80
    uint32_t al[25], ah[25];
    shake_absorb_seed_nonce<SHAKE256_RATE, 8>(al, ah, rhoprime, kappa & 0xFFFFu);
    uint2 *o = reinterpret_cast<uint2 *>(out);
#pragma unroll 1
    for (int blk = 0; blk < 5; ++blk) {
        keccak_f1600(al, ah);
#pragma unroll
        for (int w = 0; w < 17; ++w) {
            const int g = blk * 17 + w;
            if (g < LANES) o[g] = make_uint2(al[w], ah[w]);
        }
    }
}

// Bit field of `bits` bits (<= 20) starting at bit offset `bitpos` of a little-endian byte string.
__device__ __forceinline__ uint32_t get_bits(const uint8_t *p, int bitpos, int bits) {
    const int byte = bitpos >> 3, sh = bitpos & 7;
    uint32_t v = (uint32_t)p[byte] | ((uint32_t)p[byte + 1] << 8) | ((uint32_t)p[byte + 2] << 16);
    if (sh + bits > 24) v |= (uint32_t)p[byte + 3] << 24;
    return (v >> sh) & ((1u << bits) - 1u);
}

// Pack 16 consecutive values of BITS bits (16*BITS/8 bytes, a multiple of 4) into 32-bit words.
template <int BITS>
__device__ __forceinline__ void pack16_words(uint32_t *out_words, const uint32_t (&v)[16]) {
    constexpr int NW = 16 * BITS / 32;
    uint32_t w[NW];
#pragma unroll
    for (int i = 0; i < NW; ++i) w[i] = 0;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int bit = i * BITS, wi = bit >> 5, sh = bit & 31;
        w[wi] |= v[i] << sh;
        if (sh + BITS > 32) w[wi + 1] |= v[i] >> (32 - sh);
    }
#pragma unroll
    for (int i = 0; i < NW; ++i) out_words[i] = w[i];
}

// Group helpers: 16 threads, t = position, gmask = lanes of the group.
struct Group {
    int t;
    unsigned gmask;
    int32_t *sm;  // NTT_SMEM_WORDS words
};

__device__ __forceinline__ Group make_group(int32_t *smem_base, int group_in_block) {
    Group g;
    const int lane = threadIdx.x & 31;
    g.t = lane & 15;
    g.gmask = 0xFFFFu << (lane & 16);
    g.sm = smem_base + group_in_block * NTT_SMEM_WORDS;
    return g;
}

// true if any thread of the group has `pred`.
__device__ __forceinline__ bool group_any(const Group &g, bool pred) {
    return __ballot_sync(g.gmask, pred) != 0u;
}

// Reorders the group's strided slice x[i] = a[t + 16 i] into consecutive order
// y[i] = a[16 t + i] through the group's shared memory (for bit packing).
__device__ __forceinline__ void strided_to_contig(const Group &g, const int32_t (&x)[16], int32_t (&y)[16]) {
#pragma unroll
    for (int i = 0; i < 16; ++i) g.sm[g.t + 17 * i] = x[i];
    __syncwarp(g.gmask);
#pragma unroll
    for (int i = 0; i < 16; ++i) y[i] = g.sm[17 * g.t + i];
    __syncwarp(g.gmask);
}

// z coefficients a[t + 16 i] from a packed (gamma1 - z) polynomial.
template <int MODE>
__device__ __forceinline__ void unpack_z_strided(int32_t (&x)[16], const uint8_t *packed, int t) {
    constexpr int ZB = P<MODE>::Z_BITS;
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = Params<MODE>::GAMMA1 - (int32_t)get_bits(packed, (t + 16 * i) * ZB, ZB);
}

// z coefficients a[16 t + i] (the contiguous slice of group thread t) from a packed (gamma1 - z)
// polynomial whose start is 4-byte aligned: the slice is 16 * Z_BITS / 32 whole words, read as
// 32-bit loads and split with funnel shifts.
template <int MODE>
__device__ __forceinline__ void unpack_z_contig(int32_t (&x)[16], const uint8_t *packed, int t) {
    constexpr int ZB = P<MODE>::Z_BITS, NWD = ZB / 2;
    const uint32_t *w = reinterpret_cast<const uint32_t *>(packed) + NWD * t;
    uint32_t v[NWD + 1];
#pragma unroll
    for (int k = 0; k < NWD; ++k) v[k] = w[k];
    v[NWD] = 0u;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int bit = i * ZB, wi = bit >> 5, sh = bit & 31;
        const uint32_t r = __funnelshift_r(v[wi], v[wi + 1], sh) & ((1u << ZB) - 1u);
        x[i] = Params<MODE>::GAMMA1 - (int32_t)r;
    }
}

// Inverse of strided_to_contig: y[i] = a[16 t + i] -> x[i] = a[t + 16 i].
__device__ __forceinline__ void contig_to_strided(const Group &g, const int32_t (&y)[16], int32_t (&x)[16]) {
#pragma unroll
    for (int i = 0; i < 16; ++i) g.sm[17 * g.t + i] = y[i];
    __syncwarp(g.gmask);
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = g.sm[g.t + 17 * i];
    __syncwarp(g.gmask);
}

// c coefficients a[t + 16 i] from the challenge masks (occupied bits, negative bits).
__device__ __forceinline__ void challenge_strided(int32_t (&x)[16], const uint32_t *masks, int t) {
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const uint32_t occ = masks[i >> 1], neg = masks[8 + (i >> 1)];
        const int b = t + 16 * (i & 1);
        x[i] = ((occ >> b) & 1u) ? (((neg >> b) & 1u) ? -1 : 1) : 0;
    }
}

}  // namespace cudil
