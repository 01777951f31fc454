// Register-resident Keccak-f[1600] for one state per thread, plus SHAKE absorb helpers.
//
// The reference spreads one state over 25 lanes of a warp and exchanges lanes with
// __shfl_sync (include/fips202/fips202.cuh:23-69, :104-147).  Here every thread owns a whole
// state as 50 32-bit registers (lo/hi halves of the 25 lanes): theta/chi become 3-input LOP3
// operations and every 64-bit rotation two funnel shifts, with no shuffles and no idle lanes,
// so independent SHAKE streams (ExpandA's k*l entries, ExpandMask's l entries, one challenge
// hash per attempt) map one-to-one onto threads.
//
// Round constants and rotation offsets are derived from FIPS 202 (the LFSR of Algorithm 5 and
// the (t+1)(t+2)/2 rule of Algorithm 2) at compile time.
#pragma once

#include <cstdint>

#include "params.cuh"

namespace cudil {

struct KeccakTables {
    uint32_t rc_lo[24];
    uint32_t rc_hi[24];
    int rho[25];     // rotation of lane x + 5y
    int pi_src[25];  // B[dst] = rot(A[pi_src[dst]])
};

__host__ __device__ constexpr int keccak_rc_bit(unsigned t) {
    unsigned r = 1;
    if (t % 255 == 0) return 1;
    for (unsigned i = 1; i <= t % 255; i++) {
        r <<= 1;
        if (r & 0x100) r ^= 0x171;
    }
    return (int)(r & 1);
}

__host__ __device__ constexpr KeccakTables make_keccak_tables() {
    KeccakTables k{};
    for (unsigned ir = 0; ir < 24; ir++) {
        uint64_t rc = 0;
        for (unsigned j = 0; j <= 6; j++)
            if (keccak_rc_bit(j + 7 * ir)) rc |= 1ull << ((1u << j) - 1);
        k.rc_lo[ir] = (uint32_t)rc;
        k.rc_hi[ir] = (uint32_t)(rc >> 32);
    }
    for (int i = 0; i < 25; i++) k.rho[i] = 0;
    unsigned x = 1, y = 0;
    for (unsigned t = 0; t < 24; t++) {
        unsigned nx = y, ny = (2 * x + 3 * y) % 5;
        k.rho[x + 5 * y] = (int)(((t + 1) * (t + 2) / 2) % 64);
        x = nx;
        y = ny;
    }
    for (unsigned yy = 0; yy < 5; yy++)
        for (unsigned xx = 0; xx < 5; xx++) k.pi_src[xx + 5 * yy] = (int)(((xx + 3 * yy) % 5) + 5 * xx);
    return k;
}

constexpr KeccakTables kKeccak = make_keccak_tables();
static_assert(kKeccak.rc_lo[0] == 1u && kKeccak.rc_hi[0] == 0u, "keccak rc");
static_assert(kKeccak.rc_lo[23] == 0x80008008u && kKeccak.rc_hi[23] == 0x80000000u, "keccak rc");
static_assert(kKeccak.rho[1] == 1 && kKeccak.rho[24] == 14, "keccak rho");

static __constant__ KeccakTables c_keccak = make_keccak_tables();
// Compile-time copy for device code (rotation amounts and lane permutation fold to immediates).
static constexpr __device__ KeccakTables kKeccakDev = make_keccak_tables();

// 64-bit rotate-left of (h:l) by a compile-time amount (after unrolling), two funnel shifts.
__device__ __forceinline__ void rotl64(uint32_t &ol, uint32_t &oh, uint32_t l, uint32_t h, int n) {
    if (n == 0) {
        ol = l;
        oh = h;
    } else if (n < 32) {
        oh = __funnelshift_l(l, h, n);
        ol = __funnelshift_l(h, l, n);
    } else if (n == 32) {
        ol = h;
        oh = l;
    } else {
        oh = __funnelshift_l(h, l, n - 32);
        ol = __funnelshift_l(l, h, n - 32);
    }
}

// Keccak-f[1600] on a state held as lo/hi 32-bit halves.  Every array index is static after
// unrolling, so the state stays in registers.
__device__ __forceinline__ void keccak_f1600(uint32_t (&al)[25], uint32_t (&ah)[25]) {
#pragma unroll 1
    for (int r = 0; r < 24; ++r) {
        uint32_t cl[5], ch[5], bl[25], bh[25];
#pragma unroll
        for (int x = 0; x < 5; ++x) {
            cl[x] = al[x] ^ al[x + 5] ^ al[x + 10] ^ al[x + 15] ^ al[x + 20];
            ch[x] = ah[x] ^ ah[x + 5] ^ ah[x + 10] ^ ah[x + 15] ^ ah[x + 20];
        }
#pragma unroll
        for (int x = 0; x < 5; ++x) {
            uint32_t rl, rh;
            rotl64(rl, rh, cl[(x + 1) % 5], ch[(x + 1) % 5], 1);
            uint32_t dl = cl[(x + 4) % 5] ^ rl, dh = ch[(x + 4) % 5] ^ rh;
#pragma unroll
            for (int y = 0; y < 5; ++y) {
                al[x + 5 * y] ^= dl;
                ah[x + 5 * y] ^= dh;
            }
        }
#pragma unroll
        for (int i = 0; i < 25; ++i) {
            const int s = kKeccakDev.pi_src[i];
            rotl64(bl[i], bh[i], al[s], ah[s], kKeccakDev.rho[s]);
        }
#pragma unroll
        for (int y = 0; y < 5; ++y) {
#pragma unroll
            for (int x = 0; x < 5; ++x) {
                al[x + 5 * y] = bl[x + 5 * y] ^ (~bl[(x + 1) % 5 + 5 * y] & bl[(x + 2) % 5 + 5 * y]);
                ah[x + 5 * y] = bh[x + 5 * y] ^ (~bh[(x + 1) % 5 + 5 * y] & bh[(x + 2) % 5 + 5 * y]);
            }
        }
        al[0] ^= c_keccak.rc_lo[r];
        ah[0] ^= c_keccak.rc_hi[r];
    }
}

__device__ __forceinline__ void keccak_zero(uint32_t (&al)[25], uint32_t (&ah)[25]) {
#pragma unroll
    for (int i = 0; i < 25; ++i) al[i] = ah[i] = 0;
}

// Little-endian 8-byte lane from an arbitrary byte pointer; bytes at or beyond `avail` read
// as zero (avail may be >= 8 for a full lane).
__device__ __forceinline__ uint2 load_lane_bytes(const uint8_t *p, int avail) {
    uint32_t lo = 0, hi = 0;
#pragma unroll
    for (int b = 0; b < 4; ++b)
        if (b < avail) lo |= (uint32_t)p[b] << (8 * b);
#pragma unroll
    for (int b = 0; b < 4; ++b)
        if (b + 4 < avail) hi |= (uint32_t)p[b + 4] << (8 * b);
    return make_uint2(lo, hi);
}

// Lane source for a byte string whose start is 8-byte aligned.
struct AlignedBytes {
    const uint8_t *p;
    long long len;
    __device__ __forceinline__ uint2 lane(long long g) const {
        long long off = g * 8;
        if (off + 8 <= len) return *reinterpret_cast<const uint2 *>(p + off);
        return load_lane_bytes(p + off, (int)(len - off));
    }
};

// Lane source for the concatenation of two 8-byte aligned strings whose first part is a whole
// number of lanes (tr||m, mu||w1, rho'||kappa ...).
struct TwoPart {
    const uint8_t *a;
    int a_lanes;
    const uint8_t *b;
    long long b_len;
    __device__ __forceinline__ uint2 lane(long long g) const {
        if (g < a_lanes) return *reinterpret_cast<const uint2 *>(a + g * 8);
        long long off = (g - a_lanes) * 8;
        if (off + 8 <= b_len) return *reinterpret_cast<const uint2 *>(b + off);
        return load_lane_bytes(b + off, (int)(b_len - off));
    }
};

// SHAKE absorb of `total_bytes` bytes (lanes from `src`) into a zero state, with the 0x1F / 0x80
// padding applied.  The caller permutes before reading each output block.
template <int RATE, typename Src>
__device__ __forceinline__ void shake_absorb(uint32_t (&al)[25], uint32_t (&ah)[25], const Src &src,
                                             long long total_bytes) {
    constexpr int RL = RATE / 8;
    keccak_zero(al, ah);
    long long nfull = total_bytes / RATE;
    long long g = 0;
    for (long long blk = 0; blk < nfull; ++blk) {
#pragma unroll
        for (int w = 0; w < RL; ++w) {
            uint2 v = src.lane(g + w);
            al[w] ^= v.x;
            ah[w] ^= v.y;
        }
        g += RL;
        keccak_f1600(al, ah);
    }
    const int rem = (int)(total_bytes - nfull * RATE);
#pragma unroll
    for (int w = 0; w < RL; ++w) {
        uint2 v = make_uint2(0u, 0u);
        if (8 * w < rem) v = src.lane(g + w);
        if (8 * w <= rem && rem < 8 * w + 8) {
            const int sh = 8 * (rem - 8 * w);
            if (sh < 32)
                v.x ^= 0x1Fu << sh;
            else
                v.y ^= 0x1Fu << (sh - 32);
        }
        if (w == RL - 1) v.y ^= 0x80000000u;
        al[w] ^= v.x;
        ah[w] ^= v.y;
    }
}

// shake_absorb for long inputs read from global memory: the next block's lanes are loaded before
// the current block is permuted, so their latency overlaps the permutation instead of preceding
// the next one (RATE / 4 more registers live across the permutation; for kernels whose register
// budget allows it, such as the message hashes of the prehash kernels).
template <int RATE, typename Src>
__device__ __forceinline__ void shake_absorb_prefetch(uint32_t (&al)[25], uint32_t (&ah)[25], const Src &src,
                                                      long long total_bytes) {
    constexpr int RL = RATE / 8;
    keccak_zero(al, ah);
    const long long nfull = total_bytes / RATE;
    uint2 nxt[RL];
    if (nfull > 0) {
#pragma unroll
        for (int w = 0; w < RL; ++w) nxt[w] = src.lane(w);
    }
    long long g = 0;
#pragma unroll 1
    for (long long blk = 0; blk < nfull; ++blk) {
#pragma unroll
        for (int w = 0; w < RL; ++w) {
            al[w] ^= nxt[w].x;
            ah[w] ^= nxt[w].y;
        }
        g += RL;
        if (blk + 1 < nfull) {
#pragma unroll
            for (int w = 0; w < RL; ++w) nxt[w] = src.lane(g + w);
        }
        keccak_f1600(al, ah);
    }
    const int rem = (int)(total_bytes - nfull * RATE);
#pragma unroll
    for (int w = 0; w < RL; ++w) {
        uint2 v = make_uint2(0u, 0u);
        if (8 * w < rem) v = src.lane(g + w);
        if (8 * w <= rem && rem < 8 * w + 8) {
            const int sh = 8 * (rem - 8 * w);
            if (sh < 32)
                v.x ^= 0x1Fu << sh;
            else
                v.y ^= 0x1Fu << (sh - 32);
        }
        if (w == RL - 1) v.y ^= 0x80000000u;
        al[w] ^= v.x;
        ah[w] ^= v.y;
    }
}

// Seeded randomized signing: rho' = SHAKE256(seed || le64(ctr), 64), 40 bytes in one SHAKE256 block
// (seed as eight little-endian 32-bit words).
__device__ __forceinline__ void derive_rhoprime(uint2 (&out)[8], const uint32_t (&seed)[8], unsigned long long ctr) {
    uint32_t al[25], ah[25];
    keccak_zero(al, ah);
#pragma unroll
    for (int w = 0; w < 4; ++w) {
        al[w] = seed[2 * w];
        ah[w] = seed[2 * w + 1];
    }
    al[4] = (uint32_t)ctr;
    ah[4] = (uint32_t)(ctr >> 32);
    al[5] = 0x1Fu;
    ah[SHAKE256_RATE / 8 - 1] ^= 0x80000000u;
    keccak_f1600(al, ah);
#pragma unroll
    for (int w = 0; w < 8; ++w) out[w] = make_uint2(al[w], ah[w]);
}

// Absorb of a short input of IN_LANES whole lanes plus an extra 16-bit little-endian nonce
// (seed || nonce, as ExpandA/ExpandS/ExpandMask use); the input must fit one block.
template <int RATE, int IN_LANES>
__device__ __forceinline__ void shake_absorb_seed_nonce(uint32_t (&al)[25], uint32_t (&ah)[25], const uint2 (&seed)[IN_LANES],
                                                        uint32_t nonce16) {
    static_assert(IN_LANES * 8 + 2 < RATE, "single block");
    keccak_zero(al, ah);
#pragma unroll
    for (int w = 0; w < IN_LANES; ++w) {
        al[w] = seed[w].x;
        ah[w] = seed[w].y;
    }
    // bytes 8*IN_LANES, +1 = nonce, +2 = 0x1F
    al[IN_LANES] = (nonce16 & 0xFFFFu) | (0x1Fu << 16);
    ah[RATE / 8 - 1] ^= 0x80000000u;
}

}  // namespace cudil
