// Batched key generation (reference: gpu_keypair, src/keypair.cu:35-311, one warp per key).
//   k_kp_seed  one thread per key: seed (from the counter scheme of src/keypair.cu:53-59 or
//              caller-provided) -> (rho, rho', K) = SHAKE256(seed, 128)
//   k_kp_main  KPI keys per block: ExpandS streams (one thread each), eta packing and NTT(s1)
//              (16-thread groups), ExpandA streams accumulating A_ij * s1_hat_j straight into
//              t_hat (no A matrix is stored), then invNTT, + s2, Power2Round, t1/t0 packing
//   k_kp_tr    one thread per key: tr = SHAKE256(pk, 32)
#pragma once

#include "sign_kernels.cuh"

namespace cudil {

template <int MODE>
__global__ void __launch_bounds__(kBlock) k_kp_seed(uint8_t *pool, size_t pitch, int n, unsigned long long rand_index,
                                                    int seeds_given) {
    using PM = P<MODE>;
    using LY = Layout<MODE>;
    const int it = blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= n) return;
    uint8_t *row = pool + (size_t)it * pitch;
    uint32_t al[25], ah[25];
    uint2 seed[4];
    if (seeds_given) {
        // caller seed parked in sk's tr slot (written last by k_kp_tr)
        ld_lanes(seed, row + LY::KP_SK + PM::SK_TR);
    } else {
        const unsigned long long ctr = rand_index + 2ull * (unsigned long long)it + 1ull;
        keccak_zero(al, ah);
        al[0] = (uint32_t)ctr;
        ah[0] = (uint32_t)(ctr >> 32);
        al[1] = 0x1Fu;
        ah[20] ^= 0x80000000u;  // SHAKE128 rate 168 -> last lane 20
        keccak_f1600(al, ah);
#pragma unroll
        for (int w = 0; w < 4; ++w) seed[w] = make_uint2(al[w], ah[w]);
    }
    keccak_zero(al, ah);
#pragma unroll
    for (int w = 0; w < 4; ++w) {
        al[w] = seed[w].x;
        ah[w] = seed[w].y;
    }
    al[4] = 0x1Fu;
    ah[16] ^= 0x80000000u;
    keccak_f1600(al, ah);
    uint2 *pk = reinterpret_cast<uint2 *>(row + LY::KP_PK);
    uint2 *sk = reinterpret_cast<uint2 *>(row + LY::KP_SK);
    uint2 *rhop = reinterpret_cast<uint2 *>(row + LY::KP_RHOP);
#pragma unroll
    for (int w = 0; w < 4; ++w) {
        const uint2 v = make_uint2(al[w], ah[w]);
        pk[w] = v;
        sk[w] = v;
        sk[4 + w] = make_uint2(al[12 + w], ah[12 + w]);  // K
    }
#pragma unroll
    for (int w = 0; w < 8; ++w) rhop[w] = make_uint2(al[4 + w], ah[4 + w]);
}

// 16 bits-per-unit packing of 16 consecutive values of BITS bits (BITS halfwords).
template <int BITS>
__device__ __forceinline__ void pack16_halves(uint16_t *out, const uint32_t (&v)[16]) {
    uint32_t w[BITS];
#pragma unroll
    for (int i = 0; i < BITS; ++i) w[i] = 0;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int bit = i * BITS, wi = bit >> 4, sh = bit & 15;
        const uint32_t sv = v[i] << sh;  // at most BITS + 15 <= 28 bits
        w[wi] |= sv & 0xFFFFu;
        if (wi + 1 < BITS) w[wi + 1] |= (sv >> 16) & 0xFFFFu;
    }
#pragma unroll
    for (int i = 0; i < BITS; ++i) out[i] = (uint16_t)w[i];
}

template <int MODE>
struct KpSmem {
    static constexpr int K = Params<MODE>::K, L = Params<MODE>::L;
    static constexpr size_t bytes(int kpi) {
        return (size_t)kpi * (K + L) * N                      // s (int8)
               + (size_t)kpi * L * N * sizeof(int32_t)         // s1_hat
               + (size_t)kGroupsPerBlock * NTT_SMEM_WORDS * 4;  // NTT transposes
    }
};

template <int MODE, int KPI>
__global__ void __launch_bounds__(kBlock) k_kp_main(uint8_t *pool, size_t pitch, int n) {
    using PM = P<MODE>;
    using LY = Layout<MODE>;
    constexpr int K = PM::K, L = PM::L;
    extern __shared__ __align__(16) uint8_t kp_smem[];
    int32_t *s1hat = reinterpret_cast<int32_t *>(kp_smem);                         // [KPI][L][N]
    int32_t *sm = s1hat + (size_t)KPI * L * N;                                       // NTT scratch
    int8_t *s = reinterpret_cast<int8_t *>(sm + kGroupsPerBlock * NTT_SMEM_WORDS);  // [KPI][L+K][N]
    const int it0 = blockIdx.x * KPI;
    const int gi = threadIdx.x >> 4;
    Group g = make_group(sm, gi);

    // ExpandS: s1 (nonces 0..L-1) and s2 (nonces L..L+K-1)
    for (int u = threadIdx.x; u < KPI * (L + K); u += blockDim.x) {
        const int a = u / (L + K), p = u % (L + K), it = it0 + a;
        if (it >= n) continue;
        uint2 rhop[8];
        ld_lanes(rhop, pool + (size_t)it * pitch + LY::KP_RHOP);
        int8_t *sp = s + ((size_t)a * (L + K) + p) * N;
        expand_s_stream<MODE>(rhop, p, [&](int c, int32_t v) { sp[c] = (int8_t)v; });
    }
    __syncthreads();

    // eta packing of s1, s2 into sk; NTT(s1)
    for (int u = gi; u < KPI * (L + K); u += kGroupsPerBlock) {
        const int a = u / (L + K), p = u % (L + K), it = it0 + a;
        if (it >= n) continue;
        uint8_t *row = pool + (size_t)it * pitch;
        const int8_t *sp = s + ((size_t)a * (L + K) + p) * N;
        uint32_t v[16];
#pragma unroll
        for (int m = 0; m < 16; ++m) v[m] = (uint32_t)(PM::ETA - sp[16 * g.t + m]);
        uint8_t *dst = row + LY::KP_SK + PM::SK_S1 + (size_t)p * PM::POLYETA_PACKED;
        if constexpr (PM::ETA_BITS == 3)
            pack16_halves<3>(reinterpret_cast<uint16_t *>(dst + 6 * g.t), v);
        else
            pack16_words<4>(reinterpret_cast<uint32_t *>(dst + 8 * g.t), v);
        if (p < L) {
            int32_t x[16];
#pragma unroll
            for (int m = 0; m < 16; ++m) x[m] = sp[g.t + 16 * m];
            ntt16(x, g.sm, g.gmask, g.t);
            store16_contig(s1hat + ((size_t)a * L + p) * N + 16 * g.t, x);
        }
    }
    __syncthreads();

    // ExpandA fused with the matrix-vector product: t_hat_i += A_ij o s1_hat_j
    for (int u = threadIdx.x; u < KPI * K * L; u += blockDim.x) {
        const int a = u / (K * L), ij = u % (K * L), i = ij / L, j = ij % L, it = it0 + a;
        if (it >= n) continue;
        uint8_t *row = pool + (size_t)it * pitch;
        uint2 rho[4];
        ld_lanes(rho, row + LY::KP_PK);
        int32_t *acc = reinterpret_cast<int32_t *>(row + LY::KP_TACC) + (size_t)i * N;
        const int32_t *sh = s1hat + ((size_t)a * L + j) * N;
        expand_a_stream(rho, i, j, [&](int c, int32_t v) { atomicAdd(&acc[c], montmul(v, sh[c])); });
    }
    __syncthreads();

    // t = invNTT(t_hat) + s2; Power2Round; pack t1 (pk) and t0 (sk)
    for (int u = gi; u < KPI * K; u += kGroupsPerBlock) {
        const int a = u / K, i = u % K, it = it0 + a;
        if (it >= n) continue;
        uint8_t *row = pool + (size_t)it * pitch;
        const int32_t *acc = reinterpret_cast<const int32_t *>(row + LY::KP_TACC) + (size_t)i * N + 16 * g.t;
        int32_t x[16];
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = reduce32(__ldcg(acc + m));
        intt16(x, g.sm, g.gmask, g.t);
        const int8_t *s2 = s + ((size_t)a * (L + K) + L + i) * N;
        int32_t t1[16], t0[16];
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int32_t v = caddq(x[m] + s2[g.t + 16 * m]);
            t1[m] = power2round(t0[m], v);
        }
        int32_t c1[16], c0[16];
        strided_to_contig(g, t1, c1);
        strided_to_contig(g, t0, c0);
        uint32_t v1[16], v0[16];
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            v1[m] = (uint32_t)c1[m];
            v0[m] = (uint32_t)((1 << (D - 1)) - c0[m]);
        }
        pack16_words<10>(reinterpret_cast<uint32_t *>(row + LY::KP_PK + SEEDBYTES + (size_t)i * POLYT1_PACKED + 20 * g.t), v1);
        pack16_halves<13>(reinterpret_cast<uint16_t *>(row + LY::KP_SK + PM::SK_T0 + (size_t)i * POLYT0_PACKED + 26 * g.t), v0);
    }
}

template <int MODE>
__global__ void __launch_bounds__(kBlock) k_kp_tr(uint8_t *pool, size_t pitch, int n) {
    using PM = P<MODE>;
    using LY = Layout<MODE>;
    const int it = blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= n) return;
    uint8_t *row = pool + (size_t)it * pitch;
    uint32_t al[25], ah[25];
    AlignedBytes pk{row + LY::KP_PK, PM::PK_BYTES};
    shake_absorb_prefetch<SHAKE256_RATE>(al, ah, pk, PM::PK_BYTES);
    keccak_f1600(al, ah);
    uint2 *tr = reinterpret_cast<uint2 *>(row + LY::KP_SK + PM::SK_TR);
#pragma unroll
    for (int w = 0; w < 4; ++w) tr[w] = make_uint2(al[w], ah[w]);
}

}  // namespace cudil
