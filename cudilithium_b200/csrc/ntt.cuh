// Forward / inverse NTT over Z_q for one 256-coefficient polynomial held by a group of 16
// threads (16 coefficients each, two groups per warp).
//
// Arithmetic: the same Cooley-Tukey (forward) and Gentleman-Sande (inverse) butterfly network
// as the reference (src/ntt.cu:58-207, include/ntt.cuh:74-306), and the inverse ends with a
// Montgomery multiplication of every coefficient by f = 41978 (src/ntt.cu:201-205).  Two forms:
//   ntt16 / intt16   every butterfly is a +/- montmul(zeta, b) with the reference's Montgomery
//                    zetas, so outputs are bit-identical to the reference's radix-8 kernels and to
//                    the CPU oracle (key generation, the NTT microbench);
//   ntt16s / intt16s the butterflies multiply by the true zetas with precomputed quotients
//                    (shoup_mul): the same residues mod q in other representatives, for the
//                    signing and verification paths, which reduce every output before use.
//
// Layout (radix-16, one shared-memory transpose per transform instead of two):
//   forward: in  x[i] = a[t + 16 i]  -> levels len 128..16 in registers
//            transpose through shared memory (17-word padded rows, conflict-free)
//            levels len 8..1 in registers -> out x[i] = a_hat[16 t + i]
//   inverse: in  x[i] = a_hat[16 t + i] -> levels len 1..8, transpose, len 16..128, * f
//            -> out x[i] = a[t + 16 i]
// so NTT -> pointwise -> invNTT needs no extra exchange, NTT-domain data is stored in natural
// order with 64 contiguous bytes per thread (128-bit accesses) and time-domain data with 16
// consecutive words per i across the group (coalesced).
#pragma once

#include <cstdint>

#include "arith.cuh"

namespace cudil {

// Per-thread twiddles of the register-local half: 15 (zeta, zeta*qinv) pairs for each group
// position t, padded to 16 pairs (128 bytes) so a thread reads them with 8 x 128-bit loads.
struct GroupTwiddles {
    int2 fwd[16][16];  // levels len 8,4,2,1 of the forward transform
    int2 inv[16][16];  // levels len 1,2,4,8 of the inverse transform (negated zetas)
};

__host__ __device__ constexpr GroupTwiddles make_group_twiddles(const TwiddleTables &tw) {
    GroupTwiddles g{};
    for (int t = 0; t < 16; ++t) {
        int n = 0;
        // forward: len 8: zeta[16+t]; len 4: zeta[32+2t+m]; len 2: zeta[64+4t+m]; len 1: zeta[128+8t+m]
        g.fwd[t][n++] = int2{tw.zeta[16 + t], tw.zeta_q[16 + t]};
        for (int m = 0; m < 2; ++m) g.fwd[t][n++] = int2{tw.zeta[32 + 2 * t + m], tw.zeta_q[32 + 2 * t + m]};
        for (int m = 0; m < 4; ++m) g.fwd[t][n++] = int2{tw.zeta[64 + 4 * t + m], tw.zeta_q[64 + 4 * t + m]};
        for (int m = 0; m < 8; ++m) g.fwd[t][n++] = int2{tw.zeta[128 + 8 * t + m], tw.zeta_q[128 + 8 * t + m]};
        g.fwd[t][15] = int2{0, 0};
        n = 0;
        // inverse: len 1: -zeta[255-8t-m]; len 2: -zeta[127-4t-m]; len 4: -zeta[63-2t-m]; len 8: -zeta[31-t]
        for (int m = 0; m < 8; ++m) g.inv[t][n++] = int2{tw.izeta[255 - 8 * t - m], tw.izeta_q[255 - 8 * t - m]};
        for (int m = 0; m < 4; ++m) g.inv[t][n++] = int2{tw.izeta[127 - 4 * t - m], tw.izeta_q[127 - 4 * t - m]};
        for (int m = 0; m < 2; ++m) g.inv[t][n++] = int2{tw.izeta[63 - 2 * t - m], tw.izeta_q[63 - 2 * t - m]};
        g.inv[t][n++] = int2{tw.izeta[31 - t], tw.izeta_q[31 - t]};
        g.inv[t][15] = int2{0, 0};
    }
    return g;
}

static __device__ const GroupTwiddles g_group_tw = make_group_twiddles(kTwiddles);
static __device__ const GroupTwiddles g_group_tw_s = make_group_twiddles(kShoupTwiddles);
// Uniform twiddles (same for all threads of a group): zeta[1..15] and -zeta[1..15].
static __constant__ TwiddleTables c_tw = make_twiddles();
static __constant__ TwiddleTables c_tw_s = make_shoup_twiddles();

// Shared-memory words per group for the transpose (16 rows of 17).
constexpr int NTT_SMEM_WORDS = 16 * 17;

// Butterfly multiply: S = false Montgomery (twiddles in Montgomery form, the reference's exact
// representatives), S = true precomputed quotient (true twiddles, same residues).
template <bool S>
__device__ __forceinline__ int32_t bfly_mul(int32_t b, int32_t z, int32_t zq) {
    return S ? shoup_mul(b, z, zq) : montmul_pre(b, z, zq);
}

template <bool S = false>
__device__ __forceinline__ void ct_bfly(int32_t &a, int32_t &b, int32_t z, int32_t zq) {
    if constexpr (S) {
        int32_t t = bfly_mul<S>(b, z, zq);
        b = a - t;
        a = a + t;
    } else {
        // montmul_pre(b, z, zq) = hi(b z) - hi((b zq) q): the two outputs as three-input adds
        // a +/- hi(b z) -/+ hi((b zq) q), with no separate difference (same values)
        const int32_t h1 = __mulhi(b, z), h2 = __mulhi(b * zq, Q);
        b = a - h1 + h2;
        a = a + h1 - h2;
    }
}

template <bool S = false>
__device__ __forceinline__ void gs_bfly(int32_t &a, int32_t &b, int32_t z, int32_t zq) {
    int32_t t = a;
    a = t + b;
    b = bfly_mul<S>(t - b, z, zq);
}

template <bool S>
__device__ __forceinline__ const TwiddleTables &utw() {
    return S ? c_tw_s : c_tw;
}

__device__ __forceinline__ void load_tw16(int2 (&tw)[16], const int2 *src) {
    const int4 *p = reinterpret_cast<const int4 *>(src);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        int4 v = __ldg(p + i);
        tw[2 * i] = make_int2(v.x, v.y);
        tw[2 * i + 1] = make_int2(v.z, v.w);
    }
}

// Forward NTT with the thread's register-local twiddles already loaded (tw = the group position's
// row of GroupTwiddles::fwd); sm = this group's NTT_SMEM_WORDS-word region, gmask = its lanes.
template <bool S>
__device__ __forceinline__ void ntt16_tw(int32_t (&x)[16], int32_t *sm, unsigned gmask, int t, const int2 (&tw)[16]) {
    // len 128: (i, i+8), zeta[1]
#pragma unroll
    for (int i = 0; i < 8; ++i) ct_bfly<S>(x[i], x[i + 8], utw<S>().zeta[1], utw<S>().zeta_q[1]);
    // len 64: (i, i+4), zeta[2 + (i>>3)]
#pragma unroll
    for (int i = 0; i < 16; ++i)
        if (!(i & 4)) ct_bfly<S>(x[i], x[i + 4], utw<S>().zeta[2 + (i >> 3)], utw<S>().zeta_q[2 + (i >> 3)]);
    // len 32: (i, i+2), zeta[4 + (i>>2)]
#pragma unroll
    for (int i = 0; i < 16; ++i)
        if (!(i & 2)) ct_bfly<S>(x[i], x[i + 2], utw<S>().zeta[4 + (i >> 2)], utw<S>().zeta_q[4 + (i >> 2)]);
    // len 16: (i, i+1), zeta[8 + (i>>1)]
#pragma unroll
    for (int i = 0; i < 16; i += 2) ct_bfly<S>(x[i], x[i + 1], utw<S>().zeta[8 + (i >> 1)], utw<S>().zeta_q[8 + (i >> 1)]);

    // transpose: a[j] lives at sm[j + (j >> 4)]
#pragma unroll
    for (int i = 0; i < 16; ++i) sm[t + 17 * i] = x[i];
    __syncwarp(gmask);
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = sm[17 * t + i];
    __syncwarp(gmask);

    // len 8: (i, i+8), zeta[16+t]
#pragma unroll
    for (int i = 0; i < 8; ++i) ct_bfly<S>(x[i], x[i + 8], tw[0].x, tw[0].y);
    // len 4: zeta[32 + 2t + (i>>3)]
#pragma unroll
    for (int i = 0; i < 16; ++i)
        if (!(i & 4)) ct_bfly<S>(x[i], x[i + 4], tw[1 + (i >> 3)].x, tw[1 + (i >> 3)].y);
    // len 2: zeta[64 + 4t + (i>>2)]
#pragma unroll
    for (int i = 0; i < 16; ++i)
        if (!(i & 2)) ct_bfly<S>(x[i], x[i + 2], tw[3 + (i >> 2)].x, tw[3 + (i >> 2)].y);
    // len 1: zeta[128 + 8t + (i>>1)]
#pragma unroll
    for (int i = 0; i < 16; i += 2) ct_bfly<S>(x[i], x[i + 1], tw[7 + (i >> 1)].x, tw[7 + (i >> 1)].y);
}

// Forward NTT; sm = this group's NTT_SMEM_WORDS-word region, gmask = this group's lanes.
template <bool S>
__device__ __forceinline__ void ntt16_t(int32_t (&x)[16], int32_t *sm, unsigned gmask, int t) {
    int2 tw[16];
    load_tw16(tw, (S ? g_group_tw_s : g_group_tw).fwd[t]);
    ntt16_tw<S>(x, sm, gmask, t, tw);
}

// Inverse NTT including the final multiplication by f (invntt_tomont), register-local twiddles
// already loaded (tw = the group position's row of GroupTwiddles::inv).
template <bool S>
__device__ __forceinline__ void intt16_tw(int32_t (&x)[16], int32_t *sm, unsigned gmask, int t, const int2 (&tw)[16]) {
    // len 1: block 8t + (i>>1): -zeta[255 - 8t - (i>>1)]
#pragma unroll
    for (int i = 0; i < 16; i += 2) gs_bfly<S>(x[i], x[i + 1], tw[i >> 1].x, tw[i >> 1].y);
    // len 2: -zeta[127 - 4t - (i>>2)]
#pragma unroll
    for (int i = 0; i < 16; ++i)
        if (!(i & 2)) gs_bfly<S>(x[i], x[i + 2], tw[8 + (i >> 2)].x, tw[8 + (i >> 2)].y);
    // len 4: -zeta[63 - 2t - (i>>3)]
#pragma unroll
    for (int i = 0; i < 16; ++i)
        if (!(i & 4)) gs_bfly<S>(x[i], x[i + 4], tw[12 + (i >> 3)].x, tw[12 + (i >> 3)].y);
    // len 8: -zeta[31 - t]
#pragma unroll
    for (int i = 0; i < 8; ++i) gs_bfly<S>(x[i], x[i + 8], tw[14].x, tw[14].y);

#pragma unroll
    for (int i = 0; i < 16; ++i) sm[17 * t + i] = x[i];
    __syncwarp(gmask);
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = sm[t + 17 * i];
    __syncwarp(gmask);

    // len 16: (i, i+1): -zeta[15 - (i>>1)]
#pragma unroll
    for (int i = 0; i < 16; i += 2) gs_bfly<S>(x[i], x[i + 1], utw<S>().izeta[15 - (i >> 1)], utw<S>().izeta_q[15 - (i >> 1)]);
    // len 32: -zeta[7 - (i>>2)]
#pragma unroll
    for (int i = 0; i < 16; ++i)
        if (!(i & 2)) gs_bfly<S>(x[i], x[i + 2], utw<S>().izeta[7 - (i >> 2)], utw<S>().izeta_q[7 - (i >> 2)]);
    // len 64: -zeta[3 - (i>>3)]
#pragma unroll
    for (int i = 0; i < 16; ++i)
        if (!(i & 4)) gs_bfly<S>(x[i], x[i + 4], utw<S>().izeta[3 - (i >> 3)], utw<S>().izeta_q[3 - (i >> 3)]);
    // len 128: -zeta[1]
#pragma unroll
    for (int i = 0; i < 8; ++i) gs_bfly<S>(x[i], x[i + 8], utw<S>().izeta[1], utw<S>().izeta_q[1]);
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = montmul_pre(x[i], F_INV, F_INV_Q);
}

template <bool S>
__device__ __forceinline__ void intt16_t(int32_t (&x)[16], int32_t *sm, unsigned gmask, int t) {
    int2 tw[16];
    load_tw16(tw, (S ? g_group_tw_s : g_group_tw).inv[t]);
    intt16_tw<S>(x, sm, gmask, t, tw);
}

// Montgomery transforms: the reference's exact output representatives (key generation, the NTT
// microbench).
__device__ __forceinline__ void ntt16(int32_t (&x)[16], int32_t *sm, unsigned gmask, int t) { ntt16_t<false>(x, sm, gmask, t); }
__device__ __forceinline__ void intt16(int32_t (&x)[16], int32_t *sm, unsigned gmask, int t) { intt16_t<false>(x, sm, gmask, t); }
// Precomputed-quotient transforms: the same residues, cheaper butterflies (signing, verification,
// the engine's key caches -- every consumer reduces the outputs before use).
__device__ __forceinline__ void ntt16s(int32_t (&x)[16], int32_t *sm, unsigned gmask, int t) { ntt16_t<true>(x, sm, gmask, t); }
__device__ __forceinline__ void intt16s(int32_t (&x)[16], int32_t *sm, unsigned gmask, int t) { intt16_t<true>(x, sm, gmask, t); }

// Out-of-line forms of the two transforms for large kernels that call them from many places: one
// copy of each transform instead of one per call site keeps the instruction working set small.
// The 16 coefficients travel by value (registers), not through memory.
struct Coef16 {
    int32_t v[16];
};

static __device__ __noinline__ Coef16 ntt16_call(Coef16 x, int32_t *sm, unsigned gmask, int t) {
    ntt16s(x.v, sm, gmask, t);
    return x;
}

static __device__ __noinline__ Coef16 intt16_call(Coef16 x, int32_t *sm, unsigned gmask, int t) {
    intt16s(x.v, sm, gmask, t);
    return x;
}

__device__ __forceinline__ void ntt16_ool(int32_t (&x)[16], int32_t *sm, unsigned gmask, int t) {
    Coef16 c;
#pragma unroll
    for (int i = 0; i < 16; ++i) c.v[i] = x[i];
    c = ntt16_call(c, sm, gmask, t);
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = c.v[i];
}

__device__ __forceinline__ void intt16_ool(int32_t (&x)[16], int32_t *sm, unsigned gmask, int t) {
    Coef16 c;
#pragma unroll
    for (int i = 0; i < 16; ++i) c.v[i] = x[i];
    c = intt16_call(c, sm, gmask, t);
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = c.v[i];
}

// 64 contiguous bytes (natural-order NTT-domain slice 16t..16t+15) <-> registers.
__device__ __forceinline__ void load16_contig(int32_t (&x)[16], const int32_t *p) {
    const int4 *q = reinterpret_cast<const int4 *>(p);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        int4 v = q[i];
        x[4 * i] = v.x;
        x[4 * i + 1] = v.y;
        x[4 * i + 2] = v.z;
        x[4 * i + 3] = v.w;
    }
}

__device__ __forceinline__ void store16_contig(int32_t *p, const int32_t (&x)[16]) {
    int4 *q = reinterpret_cast<int4 *>(p);
#pragma unroll
    for (int i = 0; i < 4; ++i) q[i] = make_int4(x[4 * i], x[4 * i + 1], x[4 * i + 2], x[4 * i + 3]);
}

// The same 64-byte slice in shared memory with its four 16-byte chunks rotated by t, so the
// 128-bit accesses of neighbouring threads (64 bytes apart) fall into different banks.
__device__ __forceinline__ void store16_smem(int32_t *poly, const int32_t (&x)[16], int t) {
    int4 *q = reinterpret_cast<int4 *>(poly + 16 * t);
#pragma unroll
    for (int i = 0; i < 4; ++i) q[(i + t) & 3] = make_int4(x[4 * i], x[4 * i + 1], x[4 * i + 2], x[4 * i + 3]);
}

__device__ __forceinline__ void load16_smem(int32_t (&x)[16], const int32_t *poly, int t) {
    const int4 *q = reinterpret_cast<const int4 *>(poly + 16 * t);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int4 v = q[(i + t) & 3];
        x[4 * i] = v.x;
        x[4 * i + 1] = v.y;
        x[4 * i + 2] = v.z;
        x[4 * i + 3] = v.w;
    }
}

// Strided slice a[t + 16 i] <-> registers (coalesced across the group).
__device__ __forceinline__ void load16_strided(int32_t (&x)[16], const int32_t *poly, int t) {
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = poly[t + 16 * i];
}

__device__ __forceinline__ void store16_strided(int32_t *poly, const int32_t (&x)[16], int t) {
#pragma unroll
    for (int i = 0; i < 16; ++i) poly[t + 16 * i] = x[i];
}

}  // namespace cudil
