// Integer arithmetic mod q = 8380417: Montgomery multiplication, Barrett-style reduction and
// the rounding / hint functions of Dilithium v3.1.
//
// Every routine computes exactly what the reference's device helpers compute:
//   montmul ........ include/ntt.cuh:64-72 (a*b*2^-32, result in (-q, q))
//   reduce32/caddq . include/reduce.cuh:42-78
//   power2round, decompose, make_hint, use_hint ... include/rounding.cuh:22-107
//   chknorm ........ include/poly.cuh:31-54
// The twiddle table is the reference's c_zetas (src/ntt.cu:24-56), i.e. 2^32 * 1753^brv8(i)
// mod q centred; it is generated here at compile time from that definition.
#pragma once

#include <cstdint>

#include "params.cuh"

namespace cudil {

// ------------------------------------------------------------------ twiddles

struct TwiddleTables {
    int32_t zeta[N];     // zeta[i] = mont * 1753^brv8(i) mod q (centred); zeta[0] = 0
    int32_t zeta_q[N];   // zeta[i] * QINV mod 2^32
    int32_t izeta[N];    // -zeta[i]
    int32_t izeta_q[N];  // -zeta[i] * QINV mod 2^32
};

__host__ __device__ constexpr unsigned brv8(unsigned x) {
    unsigned r = 0;
    for (int i = 0; i < 8; ++i) r |= ((x >> i) & 1u) << (7 - i);
    return r;
}

__host__ __device__ constexpr int32_t mul_qinv(int32_t z) {
    return (int32_t)((uint32_t)z * (uint32_t)QINV);
}

__host__ __device__ constexpr TwiddleTables make_twiddles() {
    TwiddleTables t{};
    const uint64_t mont = (1ull << 32) % Q;
    for (int i = 0; i < N; ++i) {
        uint64_t e = brv8((unsigned)i), r = 1, b = 1753;
        while (e) {
            if (e & 1) r = r * b % Q;
            b = b * b % Q;
            e >>= 1;
        }
        r = r * mont % Q;
        int32_t z = (int32_t)(r > (uint64_t)(Q - 1) / 2 ? (int64_t)r - Q : (int64_t)r);
        if (i == 0) z = 0;
        t.zeta[i] = z;
        t.zeta_q[i] = mul_qinv(z);
        t.izeta[i] = -z;
        t.izeta_q[i] = mul_qinv(-z);
    }
    return t;
}

constexpr TwiddleTables kTwiddles = make_twiddles();
static_assert(kTwiddles.zeta[1] == 25847, "zeta table");
static_assert(kTwiddles.zeta[2] == -2608894, "zeta table");
static_assert(kTwiddles.zeta[255] == 1976782, "zeta table");

// Precomputed-quotient (Shoup) twiddles for the butterflies of the signing / verification
// transforms: the same zetas as true residues w = 1753^brv8(i) mod q (centred) with
// w_q = floor(w * 2^32 / q).  shoup_mul(b, w, w_q) = b * w - q * floor(b * w_q / 2^32) is
// congruent to b * w mod q and lies in (-q/2, 3q/2) for any 32-bit b -- one high multiply and two
// low multiply-adds instead of montmul's two high multiplies, one low multiply and a subtraction.
// The transforms built on it give the reference's residues (not its representatives), so they
// serve every path whose outputs are reduced before use; key generation and the NTT microbench,
// whose outputs are compared representative for representative, keep the Montgomery transforms.
__host__ __device__ constexpr int32_t shoup_quot(int32_t w) {
    const int64_t num = (int64_t)w * (int64_t)(1ll << 32);
    int64_t qq = num / Q;
    if (num < 0 && qq * Q != num) --qq;  // floor
    return (int32_t)qq;
}

__host__ __device__ constexpr TwiddleTables make_shoup_twiddles() {
    TwiddleTables t{};
    for (int i = 0; i < N; ++i) {
        uint64_t e = brv8((unsigned)i), r = 1, b = 1753;
        while (e) {
            if (e & 1) r = r * b % Q;
            b = b * b % Q;
            e >>= 1;
        }
        int32_t w = (int32_t)(r > (uint64_t)(Q - 1) / 2 ? (int64_t)r - Q : (int64_t)r);
        if (i == 0) w = 0;
        t.zeta[i] = w;
        t.zeta_q[i] = shoup_quot(w);
        t.izeta[i] = -w;
        t.izeta_q[i] = shoup_quot(-w);
    }
    return t;
}

constexpr TwiddleTables kShoupTwiddles = make_shoup_twiddles();

// every true twiddle times mont is the Montgomery-form twiddle (mod q)
__host__ __device__ constexpr bool shoup_matches_montgomery() {
    const int64_t mont = (int64_t)((1ull << 32) % Q);
    for (int i = 1; i < N; ++i) {
        const int64_t a = ((int64_t)kShoupTwiddles.zeta[i] * mont - (int64_t)kTwiddles.zeta[i]) % Q;
        if (a != 0) return false;
    }
    return true;
}
static_assert(shoup_matches_montgomery(), "shoup table");

// f = mont^2 / 256 (the reference's 41978) and its QINV product.
constexpr int32_t F_INV = 41978;
constexpr int32_t F_INV_Q = mul_qinv(41978);

// ------------------------------------------------------------------ montgomery

// a * b * 2^-32 mod q, |result| < q; same value as the reference's gpu_montgomery_multiply.
__device__ __forceinline__ int32_t montmul(int32_t a, int32_t b) {
    int32_t hi = __mulhi(a, b);
    int32_t t = (a * b) * QINV;
    return hi - __mulhi(t, Q);
}

// montmul(a, z) with zq = z * QINV mod 2^32 precomputed: a*zq == (a*z)*QINV mod 2^32, so the
// result is bit-identical to montmul(a, z) with one multiplication fewer.
__device__ __forceinline__ int32_t montmul_pre(int32_t a, int32_t z, int32_t zq) {
    return __mulhi(a, z) - __mulhi(a * zq, Q);
}

__device__ __forceinline__ int32_t shoup_mul(int32_t b, int32_t w, int32_t wq) {
    const int32_t t = __mulhi(b, wq);
    return (int32_t)((uint32_t)b * (uint32_t)w - (uint32_t)t * (uint32_t)Q);
}

__device__ __forceinline__ int32_t reduce32(int32_t a) {
    int32_t t = (a + (1 << 22)) >> 23;
    return a - t * Q;
}

__device__ __forceinline__ int32_t caddq(int32_t a) { return a + ((a >> 31) & Q); }

__device__ __forceinline__ int32_t power2round(int32_t &a0, int32_t a) {
    int32_t a1 = (a + (1 << (D - 1)) - 1) >> D;
    a0 = a - (a1 << D);
    return a1;
}

template <int MODE>
__device__ __forceinline__ int32_t decompose(int32_t &a0, int32_t a) {
    constexpr int G2 = Params<MODE>::GAMMA2;
    int32_t a1 = (a + 127) >> 7;
    if constexpr (G2 == (Q - 1) / 32) {
        a1 = (a1 * 1025 + (1 << 21)) >> 22;
        a1 &= 15;
    } else {
        a1 = (a1 * 11275 + (1 << 23)) >> 24;
        a1 ^= ((43 - a1) >> 31) & a1;
    }
    a0 = a - a1 * 2 * G2;
    a0 -= (((Q - 1) / 2 - a0) >> 31) & Q;
    return a1;
}

template <int MODE>
__device__ __forceinline__ unsigned make_hint(int32_t a0, int32_t a1) {
    constexpr int G2 = Params<MODE>::GAMMA2;
    return (a0 > G2 || a0 < -G2 || (a0 == -G2 && a1 != 0)) ? 1u : 0u;
}

template <int MODE>
__device__ __forceinline__ int32_t use_hint(int32_t a, unsigned hint) {
    int32_t a0;
    int32_t a1 = decompose<MODE>(a0, a);
    if (!hint) return a1;
    if constexpr (Params<MODE>::GAMMA2 == (Q - 1) / 32) {
        return (a0 > 0) ? ((a1 + 1) & 15) : ((a1 - 1) & 15);
    } else {
        if (a0 > 0) return (a1 == 43) ? 0 : a1 + 1;
        return (a1 == 0) ? 43 : a1 - 1;
    }
}

// |a| >= bound, computed without branching on the sign (include/poly.cuh:41-50).
__device__ __forceinline__ bool exceeds(int32_t a, int32_t bound) {
    int32_t t = a >> 31;
    t = a - (t & 2 * a);
    return t >= bound;
}

}  // namespace cudil
