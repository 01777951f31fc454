// Batched signing kernels (stage-by-stage).  Each kernel maps its stage onto the GPU in the shape
// that stage needs: SHAKE streams one per thread, polynomial arithmetic one per 16-thread group.
//
// Stage list (reference kernel each one replaces):
//   k_sign_prehash     mu = H(tr||m), rho' = H(K||mu)     notmp_shake_new_kernel, src/api.cu:137-152
//   k_expand_a         A_hat = ExpandA(rho)               polyvec_matrix_expand_opt_kernel, src/sign.cu:98-163
//   k_sign_unpack_ntt  s1_hat, s2_hat, t0_hat             unpack_fuse_ntt_radix2_opt_kernel, src/sign.cu:306-403
//   k_sign_expand_mask y = ExpandMask(rho', L*nonce + j)  compute_y_opt_kernel, src/sign.cu:463-526
//   k_sign_compute_w   w = invNTT(A_hat NTT(y)); w0, w1   compute_w_128t_kernel, src/sign.cu:605-685
//   k_sign_challenge   c~ = H(mu||w1), c = SampleInBall   compute_cp_kernel, src/sign.cu:687-735
//   k_sign_reject      z, r0, ct0 checks, hints, packing  rej_loop_128t_kernel, src/sign.cu:986-1196
//   k_sig_copy         move the winning attempt           sig_copy_kernel, src/sign.cu:1198-1207
#pragma once

#include "device.cuh"
#include "layout.cuh"

namespace cudil {

constexpr int kBlock = 128;             // threads per block for the SHAKE-stream kernels
constexpr int kGroupsPerBlock = 8;      // 16-thread groups per 128-thread block
constexpr int kItemBlock = 32;          // threads per block for thread-per-item kernels

// ------------------------------------------------------------------ per-item setup

// rhop_given: rho' was placed in the row by the caller (randomized signing), only mu is computed.
template <int MODE>
__global__ void __launch_bounds__(kBlock) k_sign_prehash(uint8_t *pool, size_t pitch, size_t mlen, const uint32_t *mlens,
                                                         int n, int rhop_given) {
    using LY = Layout<MODE>;
    const int it = blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= n) return;
    uint8_t *row = pool + (size_t)it * pitch;
    const size_t ml = mlens ? (size_t)mlens[it] : mlen;  // per-item length (<= mlen) when given
    uint32_t al[25], ah[25];
    TwoPart src{row + LY::SG_SK + P<MODE>::SK_TR, 4, row + LY::SG_MSG, (long long)ml};
    shake_absorb_prefetch<SHAKE256_RATE>(al, ah, src, (long long)(SEEDBYTES + ml));
    keccak_f1600(al, ah);
    uint2 mu[8];
#pragma unroll
    for (int w = 0; w < 8; ++w) mu[w] = make_uint2(al[w], ah[w]);
    uint2 *mu_out = reinterpret_cast<uint2 *>(row + LY::SG_MU);
#pragma unroll
    for (int w = 0; w < 8; ++w) mu_out[w] = mu[w];
    if (rhop_given) return;
    // rho' = SHAKE256(K || mu, 64): 96 bytes, one block
    uint2 key[4];
    ld_lanes(key, row + LY::SG_SK + P<MODE>::SK_KEY);
    keccak_zero(al, ah);
#pragma unroll
    for (int w = 0; w < 4; ++w) {
        al[w] = key[w].x;
        ah[w] = key[w].y;
    }
#pragma unroll
    for (int w = 0; w < 8; ++w) {
        al[4 + w] = mu[w].x;
        ah[4 + w] = mu[w].y;
    }
    al[12] ^= 0x1Fu;
    ah[16] ^= 0x80000000u;
    keccak_f1600(al, ah);
    uint2 *rp = reinterpret_cast<uint2 *>(row + LY::SG_RHOP);
#pragma unroll
    for (int w = 0; w < 8; ++w) rp[w] = make_uint2(al[w], ah[w]);
}

// One thread per ExpandA entry; rho at row+rho_off, A_hat (K*L polys) at row+mat_off.
template <int MODE>
__global__ void __launch_bounds__(kBlock) k_expand_a(uint8_t *pool, size_t pitch, size_t rho_off, size_t mat_off, int n) {
    constexpr int K = Params<MODE>::K, L = Params<MODE>::L, KL = K * L;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n * KL) return;
    const int it = s / KL, ij = s % KL;
    uint8_t *row = pool + (size_t)it * pitch;
    uint2 rho[4];
    ld_lanes(rho, row + rho_off);
    int32_t *out = reinterpret_cast<int32_t *>(row + mat_off) + (size_t)ij * N;
    expand_a_row(rho, ij / L, ij % L, out);
}

// The same with rho read from the packed keys (key i at keys + i * key_bytes, rho = its first 32
// bytes), so the build of a cache row's Â needs no other part of the row.
template <int MODE>
__global__ void __launch_bounds__(kBlock) k_expand_a_keys(const uint8_t *keys, size_t key_bytes, uint8_t *rows, size_t pitch,
                                                          size_t mat_off, int n) {
    constexpr int K = Params<MODE>::K, L = Params<MODE>::L, KL = K * L;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n * KL) return;
    const int it = s / KL, ij = s % KL;
    const uint8_t *key = keys + (size_t)it * key_bytes;
    uint2 rho[4];
    if ((reinterpret_cast<uintptr_t>(key) & 7u) == 0u) {
        ld_lanes(rho, key);
    } else {
#pragma unroll
        for (int w = 0; w < 4; ++w) rho[w] = load_lane_bytes(key + 8 * w, 8);
    }
    int32_t *out = reinterpret_cast<int32_t *>(rows + (size_t)it * pitch + mat_off) + (size_t)ij * N;
    expand_a_row(rho, ij / L, ij % L, out);
}

// One 16-thread group per secret polynomial: unpack (eta / 13-bit) and forward NTT.
template <int MODE>
__global__ void __launch_bounds__(kBlock) k_sign_unpack_ntt(uint8_t *pool, size_t pitch, size_t mlen, int n) {
    using PM = P<MODE>;
    using LY = Layout<MODE>;
    constexpr int K = PM::K, L = PM::L, NP = L + 2 * K;
    __shared__ int32_t sm[kGroupsPerBlock * NTT_SMEM_WORDS];
    const int gid = (blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    const int it = gid / NP, p = gid % NP;
    if (it >= n) return;
    Group g = make_group(sm, threadIdx.x >> 4);
    uint8_t *row = pool + (size_t)it * pitch;
    const uint8_t *sk = row + LY::SG_SK;
    int32_t x[16];
    size_t dst;
    if (p < L + K) {
        const uint8_t *src = sk + PM::SK_S1 + (size_t)p * PM::POLYETA_PACKED;
#pragma unroll
        for (int i = 0; i < 16; ++i) x[i] = PM::ETA - (int32_t)get_bits(src, (g.t + 16 * i) * PM::ETA_BITS, PM::ETA_BITS);
        dst = (p < L) ? LY::sg_s1(mlen) + (size_t)p * LY::POLY : LY::sg_s2(mlen) + (size_t)(p - L) * LY::POLY;
    } else {
        const uint8_t *src = sk + PM::SK_T0 + (size_t)(p - L - K) * POLYT0_PACKED;
#pragma unroll
        for (int i = 0; i < 16; ++i) x[i] = (1 << (D - 1)) - (int32_t)get_bits(src, (g.t + 16 * i) * 13, 13);
        dst = LY::sg_t0(mlen) + (size_t)(p - L - K) * LY::POLY;
    }
    ntt16s(x, g.sm, g.gmask, g.t);
    store16_contig(reinterpret_cast<int32_t *>(row + dst) + 16 * g.t, x);
}

// ------------------------------------------------------------------ per-attempt stages

// exec_lut entry = (item << 16) | nonce, as the reference's task_lut (src/api.cu:221-230).
template <int MODE>
__global__ void __launch_bounds__(kBlock) k_sign_expand_mask(const uint8_t *sign_pool, size_t sp, uint8_t *temp_pool,
                                                             size_t tp, const uint32_t *exec_lut, int nexec, int nitems) {
    using LY = Layout<MODE>;
    constexpr int L = Params<MODE>::L;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nexec * L) return;
    const int e = s / L, j = s % L;
    const uint32_t info = exec_lut[e];
    const uint32_t item = info >> 16, nonce = info & 0xFFFFu;
    if (!bc_ok(item < (uint32_t)nitems, BC_STAGE_ITEM)) return;
    uint2 rhop[8];
    ld_lanes(rhop, sign_pool + (size_t)item * sp + LY::SG_RHOP);
    expand_mask_stream<MODE>(temp_pool + (size_t)e * tp + LY::TP_Y + (size_t)j * P<MODE>::POLYZ_PACKED, rhop,
                             (uint32_t)(L * nonce + j));
}

// AW attempts per 128-thread block: NTT(y_j) into shared memory, then one group per row i
// computes w_i = invNTT(sum_j A_ij * y_hat_j), Decompose, w0 and packed w1.
template <int MODE, int AW>
__global__ void __launch_bounds__(kBlock) k_sign_compute_w(const uint8_t *sign_pool, size_t sp, size_t mlen, uint8_t *temp_pool,
                                                           size_t tp, const uint32_t *exec_lut, int nexec, int nitems) {
    using PM = P<MODE>;
    using LY = Layout<MODE>;
    constexpr int K = PM::K, L = PM::L;
    __shared__ __align__(16) int32_t s_yhat[AW][L][N];
    __shared__ int32_t sm[kGroupsPerBlock * NTT_SMEM_WORDS];
    const int gi = threadIdx.x >> 4;
    Group g = make_group(sm, gi);
    const int e0 = blockIdx.x * AW;
    for (int u = gi; u < AW * L; u += kGroupsPerBlock) {
        const int a = u / L, j = u % L, e = e0 + a;
        if (e >= nexec) continue;
        int32_t x[16];
        unpack_z_strided<MODE>(x, temp_pool + (size_t)e * tp + LY::TP_Y + (size_t)j * PM::POLYZ_PACKED, g.t);
        ntt16s(x, g.sm, g.gmask, g.t);
        store16_smem(&s_yhat[a][j][0], x, g.t);
    }
    __syncthreads();
    for (int u = gi; u < AW * K; u += kGroupsPerBlock) {
        const int a = u / K, i = u % K, e = e0 + a;
        if (e >= nexec) continue;
        const uint32_t item = exec_lut[e] >> 16;
        if (!bc_ok(item < (uint32_t)nitems, BC_STAGE_ITEM)) continue;
        const int32_t *mat = reinterpret_cast<const int32_t *>(sign_pool + (size_t)item * sp + LY::sg_mat(mlen)) + (size_t)i * L * N;
        int32_t acc[16];
#pragma unroll
        for (int m = 0; m < 16; ++m) acc[m] = 0;
#pragma unroll
        for (int j = 0; j < L; ++j) {
            int32_t av[16], yv[16];
            load16_contig(av, mat + (size_t)j * N + 16 * g.t);
            load16_smem(yv, &s_yhat[a][j][0], g.t);
#pragma unroll
            for (int m = 0; m < 16; ++m) acc[m] += montmul(av[m], yv[m]);
        }
#pragma unroll
        for (int m = 0; m < 16; ++m) acc[m] = reduce32(acc[m]);
        intt16s(acc, g.sm, g.gmask, g.t);
        uint8_t *trow = temp_pool + (size_t)e * tp;
        int32_t *w0 = reinterpret_cast<int32_t *>(trow + LY::TP_W0) + (size_t)i * N;
        int32_t w1[16];
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            int32_t a0;
            w1[m] = decompose<MODE>(a0, caddq(acc[m]));
            w0[g.t + 16 * m] = a0;
        }
        int32_t w1c[16];
        strided_to_contig(g, w1, w1c);
        uint32_t v[16];
#pragma unroll
        for (int m = 0; m < 16; ++m) v[m] = (uint32_t)w1c[m];
        pack16_words<PM::W1_BITS>(reinterpret_cast<uint32_t *>(trow + LY::TP_W1P + (size_t)i * PM::POLYW1_PACKED + g.t * 2 * PM::W1_BITS), v);
    }
}

// SampleInBall(c~) (src/sign.cu:767-787), one thread per challenge.  The squeezed block (34
// words) and the result (two 256-bit masks: non-zero positions, negative positions; 16 words) live
// in shared memory interleaved across the threads of the block -- word k of this thread at
// [k * STRIDE] -- so the dynamically indexed accesses of neighbouring threads hit distinct banks.
template <int TAU, int STRIDE>
__device__ __forceinline__ void sample_in_ball(const uint2 (&ct)[4], uint32_t *blkw, uint32_t *mask) {
    uint32_t al[25], ah[25];
    keccak_zero(al, ah);
#pragma unroll
    for (int w = 0; w < 4; ++w) {
        al[w] = ct[w].x;
        ah[w] = ct[w].y;
    }
    al[4] = 0x1Fu;
    ah[16] ^= 0x80000000u;
    keccak_f1600(al, ah);
#pragma unroll
    for (int w = 0; w < 17; ++w) {
        blkw[(2 * w) * STRIDE] = al[w];
        blkw[(2 * w + 1) * STRIDE] = ah[w];
    }
    uint32_t sl = al[0], sh = ah[0];
#pragma unroll
    for (int k = 0; k < 16; ++k) mask[k * STRIDE] = 0;
    int pos = 8;
#pragma unroll 1
    for (int i = N - TAU; i < N; ++i) {
        uint32_t b;
        do {
            if (pos >= SHAKE256_RATE) {
                keccak_f1600(al, ah);
#pragma unroll
                for (int w = 0; w < 17; ++w) {
                    blkw[(2 * w) * STRIDE] = al[w];
                    blkw[(2 * w + 1) * STRIDE] = ah[w];
                }
                pos = 0;
            }
            b = (blkw[(pos >> 2) * STRIDE] >> (8 * (pos & 3))) & 0xFFu;
            ++pos;
        } while (b > (uint32_t)i);
        const uint32_t wb = b >> 5, bb = 1u << (b & 31);
        const uint32_t wi = (uint32_t)i >> 5, bi = 1u << (i & 31);
        uint32_t *occ_b = mask + wb * STRIDE, *neg_b = mask + (8 + wb) * STRIDE;
        uint32_t *occ_i = mask + wi * STRIDE, *neg_i = mask + (8 + wi) * STRIDE;
        const uint32_t ob = *occ_b & bb, nb = *neg_b & bb;
        // c[i] = c[b]
        *occ_i = ob ? (*occ_i | bi) : (*occ_i & ~bi);
        *neg_i = nb ? (*neg_i | bi) : (*neg_i & ~bi);
        // c[b] = 1 - 2 * (signs & 1)
        *occ_b |= bb;
        *neg_b = (sl & 1u) ? (*neg_b | bb) : (*neg_b & ~bb);
        sl = (sl >> 1) | (sh << 31);
        sh >>= 1;
    }
}

// Thread-per-item kernels run TB = kItemBlock threads per block so that batches of a few thousand
// items still spread over every SM.
template <int MODE, int TB = kItemBlock>
__global__ void __launch_bounds__(TB) k_sign_challenge(const uint8_t *sign_pool, size_t sp, uint8_t *temp_pool, size_t tp,
                                                       const uint32_t *exec_lut, int nexec, int nitems) {
    using PM = P<MODE>;
    using LY = Layout<MODE>;
    __shared__ uint32_t s_blk[2 * 17][TB];
    __shared__ uint32_t s_mask[16][TB];
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nexec) return;
    const uint32_t item = exec_lut[e] >> 16;
    if (!bc_ok(item < (uint32_t)nitems, BC_STAGE_ITEM)) return;
    uint8_t *trow = temp_pool + (size_t)e * tp;
    uint32_t al[25], ah[25];
    TwoPart src{sign_pool + (size_t)item * sp + LY::SG_MU, 8, trow + LY::TP_W1P, PM::W1PACKED_BYTES};
    shake_absorb<SHAKE256_RATE>(al, ah, src, CRHBYTES + PM::W1PACKED_BYTES);
    keccak_f1600(al, ah);
    uint2 ct[4];
#pragma unroll
    for (int w = 0; w < 4; ++w) ct[w] = make_uint2(al[w], ah[w]);
    uint2 *sig_ct = reinterpret_cast<uint2 *>(trow + LY::TP_SIG);
#pragma unroll
    for (int w = 0; w < 4; ++w) sig_ct[w] = ct[w];
    uint32_t *mask = &s_mask[0][threadIdx.x];
    sample_in_ball<PM::TAU, TB>(ct, &s_blk[0][threadIdx.x], mask);
    uint4 *mo = reinterpret_cast<uint4 *>(trow + LY::TP_CMASK);
#pragma unroll
    for (int k = 0; k < 4; ++k)
        mo[k] = make_uint4(mask[(4 * k) * TB], mask[(4 * k + 1) * TB], mask[(4 * k + 2) * TB], mask[(4 * k + 3) * TB]);
}

// One warp per attempt: c_hat = NTT(c); r0 = w0 - c*s2, z = y + c*s1 and c*t0 (norm checks);
// MakeHint (at most OMEGA, positions in ascending order).  The two 16-thread groups of the warp
// take the attempt's polynomials in pairs (poly 2p + half), so they follow the same control flow
// and a rejection ends the attempt for the whole warp.  On acceptance the temp row holds the
// complete signature and done[e] = 1 (src/sign.cu:1010-1195).
template <int MODE>
__global__ void __launch_bounds__(kBlock, 4) k_sign_reject(const uint8_t *sign_pool, size_t sp, size_t mlen, uint8_t *temp_pool,
                                                        size_t tp, const uint32_t *exec_lut, uint8_t *done, int nexec,
                                                        int nitems) {
    using PM = P<MODE>;
    using LY = Layout<MODE>;
    constexpr int K = PM::K, L = PM::L, OMEGA = PM::OMEGA;
    __shared__ int32_t sm[kGroupsPerBlock * NTT_SMEM_WORDS];
    const int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (e >= nexec) return;  // (the same for the whole warp)
    Group g = make_group(sm, threadIdx.x >> 4);
    const int lane = threadIdx.x & 31, lane_off = lane & 16, half = lane_off >> 4;
    const uint32_t item = exec_lut[e] >> 16;
    if (!bc_ok(item < (uint32_t)nitems, BC_STAGE_ITEM)) return;
    const uint8_t *srow = sign_pool + (size_t)item * sp;
    uint8_t *trow = temp_pool + (size_t)e * tp;

    uint32_t masks[16];
    {
        const uint4 *mi = reinterpret_cast<const uint4 *>(trow + LY::TP_CMASK);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            uint4 v = mi[k];
            masks[4 * k] = v.x;
            masks[4 * k + 1] = v.y;
            masks[4 * k + 2] = v.z;
            masks[4 * k + 3] = v.w;
        }
    }
    // both groups transform c (same data, same instructions)
    int32_t ch[16];
    challenge_strided(ch, masks, g.t);
    ntt16s(ch, g.sm, g.gmask, g.t);

    // Acceptance needs every check to pass (src/sign.cu:1026-1144 checks z, then r0, then ct0);
    // here the most selective runs first: pair steps of the r0_i (r0 replaces w0 in the temp row,
    // for the hints), then of the z_j, then of the ct0_i with the hints.  K is even for every
    // parameter set; L is odd for two of them, so the last z pair may leave the second group
    // without a polynomial (it transforms zeros and stores nothing).  One inverse-NTT call site;
    // the next step's key rows load while the current one transforms.
    const int32_t *s1 = reinterpret_cast<const int32_t *>(srow + LY::sg_s1(mlen));
    const int32_t *s2 = reinterpret_cast<const int32_t *>(srow + LY::sg_s2(mlen));
    const int32_t *t0 = reinterpret_cast<const int32_t *>(srow + LY::sg_t0(mlen));
    constexpr int PR = K / 2, PZ = (L + 1) / 2, NSTEP = 2 * PR + PZ;
    auto operand = [&](int step) -> const int32_t * {
        if (step < PR) return s2 + (size_t)(2 * step + half) * N;
        if (step < PR + PZ) {
            const int j = 2 * (step - PR) + half;
            return s1 + (size_t)(j < L ? j : L - 1) * N;
        }
        return t0 + (size_t)(2 * (step - PR - PZ) + half) * N;
    };
    uint8_t *hs = trow + LY::TP_SIG + PM::SIG_H;
    int cnt = 0;
    int32_t nx[16];
    load16_contig(nx, operand(0) + 16 * g.t);
#pragma unroll 1
    for (int step = 0; step < NSTEP; ++step) {
        const bool is_r0 = step < PR, is_z = !is_r0 && step < PR + PZ;
        const int k = 2 * (is_r0 ? step : (is_z ? step - PR : step - PR - PZ)) + half;  // i, or j for z
        const bool act = !is_z || k < L;
        int32_t x[16];
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = act ? montmul(ch[m], nx[m]) : 0;
        if (step + 1 < NSTEP) load16_contig(nx, operand(step + 1) + 16 * g.t);
        intt16s(x, g.sm, g.gmask, g.t);
        bool bad = false;
        if (is_z) {
            int32_t y[16];
            unpack_z_strided<MODE>(y, trow + LY::TP_Y + (size_t)(act ? k : 0) * PM::POLYZ_PACKED, g.t);
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                x[m] = reduce32(x[m] + (act ? y[m] : 0));
                bad |= act && exceeds(x[m], PM::GAMMA1 - PM::BETA);
            }
            if (__ballot_sync(0xFFFFFFFFu, bad)) return;
            int32_t zc[16];
            strided_to_contig(g, x, zc);
            if (act) {
                uint32_t v[16];
#pragma unroll
                for (int m = 0; m < 16; ++m) v[m] = (uint32_t)(PM::GAMMA1 - zc[m]);
                pack16_words<PM::Z_BITS>(
                    reinterpret_cast<uint32_t *>(trow + LY::TP_SIG + PM::SIG_Z + (size_t)k * PM::POLYZ_PACKED + g.t * 2 * PM::Z_BITS), v);
            }
        } else if (is_r0) {
            int32_t *w0 = reinterpret_cast<int32_t *>(trow + LY::TP_W0) + (size_t)k * N;
            int32_t r0[16];
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                r0[m] = reduce32(w0[g.t + 16 * m] - x[m]);
                bad |= exceeds(r0[m], PM::GAMMA2 - PM::BETA);
            }
            if (__ballot_sync(0xFFFFFFFFu, bad)) return;
#pragma unroll
            for (int m = 0; m < 16; ++m) w0[g.t + 16 * m] = r0[m];
        } else {
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                x[m] = reduce32(x[m]);
                bad |= exceeds(x[m], PM::GAMMA2);
            }
            if (__ballot_sync(0xFFFFFFFFu, bad)) return;
            const int32_t *r0 = reinterpret_cast<const int32_t *>(trow + LY::TP_W0) + (size_t)k * N;
            const uint8_t *w1p = trow + LY::TP_W1P + (size_t)k * PM::POLYW1_PACKED;
            // hint bits of poly k: bit m of hb = hint of coefficient t + 16 m
            unsigned hb = 0;
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                const int32_t w1 = (int32_t)get_bits(w1p, (g.t + 16 * m) * PM::W1_BITS, PM::W1_BITS);
                hb |= make_hint<MODE>(r0[g.t + 16 * m] + x[m], w1) << m;
            }
            // hint counts of both polynomials of the pair, then the positions in ascending
            // coefficient order: poly 2p first, then poly 2p + 1
            int tot = __popc(hb);
#pragma unroll
            for (int o = 8; o >= 1; o >>= 1) tot += __shfl_xor_sync(0xFFFFFFFFu, tot, o);
            const int tot0 = __shfl_sync(0xFFFFFFFFu, tot, 0), tot1 = __shfl_sync(0xFFFFFFFFu, tot, 16);
            if (cnt + tot0 + tot1 > OMEGA) return;
            int idx = cnt + (half ? tot0 : 0);
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                const unsigned bit = (hb >> m) & 1u;
                const unsigned bal = (__ballot_sync(0xFFFFFFFFu, bit) >> lane_off) & 0xFFFFu;
                if (bit) hs[idx + __popc(bal & ((1u << g.t) - 1u))] = (uint8_t)(g.t + 16 * m);
                idx += __popc(bal);
            }
            if (g.t == 0) hs[OMEGA + k] = (uint8_t)(cnt + (half ? tot0 + tot1 : tot0));
            cnt += tot0 + tot1;
        }
    }
    for (int q = cnt + lane; q < OMEGA; q += 32) hs[q] = 0;
    if (lane == 0) done[e] = 1;
}

struct CopyEntry {
    size_t exec_idx;
    size_t sign_idx;
};

template <int MODE>
__global__ void k_sig_copy(uint8_t *sign_pool, size_t sp, const uint8_t *temp_pool, size_t tp, const CopyEntry *lut,
                           size_t nexec, size_t nitems) {
    const CopyEntry e = lut[blockIdx.x];
    if (!bc_ok(e.exec_idx < nexec && e.sign_idx < nitems, BC_COPY_ENTRY)) return;
    const uint8_t *src = temp_pool + e.exec_idx * tp + Layout<MODE>::TP_SIG;
    uint8_t *dst = sign_pool + e.sign_idx * sp + Layout<MODE>::SG_SIG;
    for (int i = threadIdx.x; i < P<MODE>::SIG_BYTES; i += blockDim.x) dst[i] = src[i];
}

}  // namespace cudil
