// Asynchronous persistent signer: the same work queue as k_fused_sign (static item ownership per
// block, per-item next-nonce / in-flight counters, smallest accepted nonce wins), scheduled without
// block-wide barriers.
//
// Every block keeps NS attempt slots.  A slot moves through
//     FREE -> MASK -> W -> CH -> REJ -> FREE
// where MASK needs ExpandMask (L Keccak streams), W needs w = invNTT(A_hat NTT(y)) with Decompose
// and the w1 packing, CH needs c~ = H(mu || w1) and SampleInBall, REJ needs the rejection checks,
// hints and, when accepted, publication.  The states live in shared memory; a warp with nothing in
// hand scans them, takes ready slots with an atomicCAS (state -> BUSY), does the job and hands the
// slot to the next state, so a warp never waits for another one to finish a phase:
//   * Keccak jobs are lane-parallel: a warp takes up to 32 / L slots for ExpandMask (one lane per
//     (slot, j) stream) or up to 32 slots for the challenge (one lane per slot);
//   * NTT jobs are warp-per-attempt: the warp's two 16-thread groups work on two polynomials of the
//     same attempt (y_j / rows i / z_j / (r0_i, ct0_i) pairs), so both halves follow the same
//     control flow and a rejection ends the job for the whole warp;
//   * claiming (one warp at a time) turns FREE slots into MASK slots for the block's pending items,
//     at most D attempts in flight per item, D = spec_slots / pending clamped to [1, 16];
//   * an attempt whose nonce is above an already accepted nonce of its item is dropped at the next
//     job boundary (it can no longer be the winner).
// Every wait is bounded (idle polls, the per-item publication lock); running out sets an error bit
// in the queue block and the block exits.
#pragma once

#include "fused_kernels.cuh"

namespace cudil {

enum : unsigned { AS_FREE = 0, AS_MASK = 1, AS_W = 2, AS_CH = 3, AS_REJ = 4, AS_BUSY = 5 };

template <int MODE, int THREADS, int NS>
struct AsyncSignSmem {
    using PM = P<MODE>;
    static constexpr int NW = THREADS / 32;
    // per-warp work area: NTT jobs use y_hat (L polynomials) + two transpose areas; Keccak jobs use
    // the SampleInBall scratch of 32 lanes (34 block words + 16 mask words each, interleaved)
    static constexpr size_t WA_NTT = (size_t)PM::L * N * 4 + 2 * NTT_SMEM_WORDS * 4;
    static constexpr size_t WA_KEC = (size_t)(34 + 16) * 32 * 4;
    static constexpr size_t WA_CLAIM = (size_t)NS * 4;
    static constexpr size_t WA0 = WA_NTT > WA_KEC ? WA_NTT : WA_KEC;
    static constexpr size_t WA = ((WA0 > WA_CLAIM ? WA0 : WA_CLAIM) + 15) / 16 * 16;
    // control: s_item[NS], s_nonce[NS], s_state[NS], 16 counters
    static constexpr size_t CTRL = ((size_t)NS * 12 + 64 + 15) / 16 * 16;
    static constexpr size_t BYTES = CTRL + (size_t)NW * WA;
};

constexpr unsigned kAsyncIdleLimit = 1u << 21;  // default idle polls (x ~0.3 us) before a block gives up

template <int MODE, int THREADS, int NS>
__global__ void __launch_bounds__(THREADS, (THREADS >= 512) ? 1 : 512 / THREADS) k_fused_sign_async(FusedSignArgs arg) {
    using PM = P<MODE>;
    using C = Cache<MODE>;
    using SM = AsyncSignSmem<MODE, THREADS, NS>;
    constexpr int K = PM::K, L = PM::L, OMEGA = PM::OMEGA;
    constexpr int MS = 32 / L;  // slots per ExpandMask job
    static_assert(NS % 32 == 0 && NS >= 64, "slot count");
    enum { CT_PEND = 0, CT_LOCK, CT_ERR, CT_SCAN, CT_INTT, CT_PREF };
    extern __shared__ __align__(16) uint8_t as_smem[];
    unsigned *s_item = reinterpret_cast<unsigned *>(as_smem);
    unsigned *s_nonce = s_item + NS;
    unsigned *s_state = s_nonce + NS;
    unsigned *s_ctl = s_state + NS;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, half = lane >> 4, lane_off = lane & 16;
    uint8_t *wa = as_smem + SM::CTRL + (size_t)warp * SM::WA;
    FusedQueue *q = arg.q;
    const unsigned n = q->n, grid = gridDim.x, b0 = blockIdx.x;
    const unsigned n_own = (b0 < n) ? (n - b0 + grid - 1) / grid : 0u;
    uint8_t *my_slots = arg.scratch + (size_t)blockIdx.x * NS * C::SLOT;
    auto slot_ptr = [&](unsigned s) { return my_slots + (size_t)s * C::SLOT; };
    auto superseded = [&](unsigned item, unsigned nonce) { return __ldcg(arg.best + item) < nonce; };

    for (int s = tid; s < NS; s += THREADS) s_state[s] = AS_FREE;
    if (tid < 16) s_ctl[tid] = 0;
    __syncthreads();
    if (tid == 0) s_ctl[CT_PEND] = n_own;
    __syncthreads();

    Group g;
    g.t = lane & 15;
    g.gmask = 0xFFFFu << lane_off;
    const unsigned FULL = 0xFFFFFFFFu;

    // hand a slot to its next state (after this warp's writes of the slot data are visible)
    auto publish = [&](unsigned s, unsigned st) {
        __threadfence_block();
        atomicExch(&s_state[s], st);
    };
    // end of an attempt: slot back to FREE, one in-flight attempt less for the item
    auto retire = [&](unsigned s, unsigned item) {
        atomicSub(arg.inflight + item, 1u);
        publish(s, AS_FREE);
    };

    // ---------------------------------------------------------------- claim (one warp at a time)
    // Grabs the FREE slots, gives pending items their next nonces (pass p gives one more attempt to
    // items with at most p in flight, p < D) and hands the filled slots to MASK.  Returns the number
    // of attempts issued.
    const unsigned target = (arg.spec_slots && arg.spec_slots < (unsigned)NS) ? arg.spec_slots : (unsigned)NS;
    auto claim = [&]() -> unsigned {
        unsigned *grab = reinterpret_cast<unsigned *>(wa);
        unsigned ng = 0;
#pragma unroll 1
        for (int base = 0; base < NS; base += 32) {
            const unsigned s = (unsigned)(base + lane);
            bool got = false;
            if (*reinterpret_cast<volatile unsigned *>(&s_state[s]) == AS_FREE)
                got = (atomicCAS(&s_state[s], AS_FREE, AS_BUSY) == AS_FREE);
            const unsigned bal = __ballot_sync(FULL, got);
            if (got) grab[ng + __popc(bal & ((1u << lane) - 1u))] = s;
            ng += __popc(bal);
        }
        __syncwarp();
        const unsigned pend = *reinterpret_cast<volatile unsigned *>(&s_ctl[CT_PEND]);
        unsigned D = 1;
        if (pend) {
            const unsigned t = target / pend;
            D = t < 1u ? 1u : (t > 16u ? 16u : t);
        }
        unsigned filled = 0;  // grab[0, filled) hold an attempt (s_item set) or a failed placement
        const unsigned start = s_ctl[CT_SCAN];
#pragma unroll 1
        for (unsigned pass = 0; pass < D && filled < ng; ++pass) {
#pragma unroll 1
            for (unsigned k0 = 0; k0 < n_own && filled < ng; k0 += 32) {
                unsigned k = start + k0 + lane;
                if (k >= n_own) k -= n_own;
                const unsigned i = b0 + k * grid;
                // a lane with k0 + lane < n_own has k < n_own after the wrap (start < n_own), so i is an
                // owned item; its two loads issue together (one round trip, not two dependent ones)
                const bool valid = (k0 + lane) < n_own;
                unsigned bi = 0u, fi = 0u;
                if (valid) {
                    bi = __ldcg(arg.best + i);
                    fi = __ldcg(arg.inflight + i);
                }
                const bool ok = valid && bi == 0xFFFFFFFFu && fi <= pass;
                const unsigned bal = __ballot_sync(FULL, ok);
                const unsigned pos = filled + __popc(bal & ((1u << lane) - 1u));
                if (ok && pos < ng) {
                    const unsigned sl = grab[pos];
                    const unsigned nn = atomicAdd(arg.next_nonce + i, 1u);
                    if (nn < arg.nonce_limit) {
                        atomicAdd(arg.inflight + i, 1u);
                        s_item[sl] = i;
                        s_nonce[sl] = nn;
                    } else {
                        // every nonce used without acceptance: no attempt; the first lane to get here
                        // marks the item finished (error bit 1) so that the block can exit
                        s_item[sl] = 0xFFFFFFFFu;
                        if (atomicCAS(arg.best + i, 0xFFFFFFFFu, kNonceExhausted) == 0xFFFFFFFFu) {
                            atomicOr(&q->error, 2u);
                            atomicSub(&s_ctl[CT_PEND], 1u);
                        }
                    }
                }
                filled = min(ng, filled + __popc(bal));
            }
        }
        if (lane == 0) s_ctl[CT_SCAN] = n_own ? (start + 32u) % n_own : 0u;
        __threadfence_block();
        __syncwarp();
        unsigned issued = 0;
        for (unsigned k = lane; k < ng; k += 32) {
            const unsigned sl = grab[k];
            const bool real = k < filled && s_item[sl] != 0xFFFFFFFFu;
            issued += real ? 1u : 0u;
            atomicExch(&s_state[sl], real ? (unsigned)AS_MASK : (unsigned)AS_FREE);
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) issued += __shfl_xor_sync(FULL, issued, o);
        if (lane == 0 && issued) atomicAdd(&q->attempts, (unsigned long long)issued);
        __syncwarp();
        return issued;
    };

    // ---------------------------------------------------------------- ExpandMask (lane per stream)
    auto mask_job = [&](const unsigned (&sl)[MS], int cnt) {
        const int a = lane / L, j = lane % L;
        const bool act = a < cnt;
        unsigned s = 0, item = 0, nonce = 0;
        if (act) {
            s = sl[a];
            item = s_item[s];
            nonce = s_nonce[s];
        }
        // one decision per slot (its j == 0 lane), shared by the slot's L lanes
        bool drop = act && j == 0 && superseded(item, nonce);
        drop = __shfl_sync(FULL, drop, min(a * L, 31));
        drop = drop && act;
        if (act && !drop) {
            uint2 rhop[8];
            ld_lanes(rhop, arg.items + (size_t)item * C::ITEM_BYTES + 64);
            expand_mask_stream<MODE>(slot_ptr(s) + C::SL_Y + (size_t)j * PM::POLYZ_PACKED, rhop, (uint32_t)(L * nonce + j));
        }
        __threadfence_block();
        __syncwarp();
        if (act && j == 0) {
            if (drop)
                retire(s, item);
            else
                publish(s, AS_W);
        }
        __syncwarp();
    };

    // ---------------------------------------------------------------- challenge (lane per slot)
    auto challenge_job = [&](unsigned s, bool act) {
        uint32_t *blkw = reinterpret_cast<uint32_t *>(wa) + lane;
        uint32_t *mask = reinterpret_cast<uint32_t *>(wa) + 34 * 32 + lane;
        unsigned item = 0, nonce = 0;
        if (act) {
            item = s_item[s];
            nonce = s_nonce[s];
            act = bc_ok(item < n, BC_SIGN_SLOT);
        }
        const bool drop = act && superseded(item, nonce);
        if (act && !drop) {
            uint8_t *slot = slot_ptr(s);
            uint32_t al[25], ah[25];
            TwoPart src{arg.items + (size_t)item * C::ITEM_BYTES, 8, slot + C::SL_W1P, PM::W1PACKED_BYTES};
            shake_absorb<SHAKE256_RATE>(al, ah, src, CRHBYTES + PM::W1PACKED_BYTES);
            keccak_f1600(al, ah);
            uint2 ct[4];
#pragma unroll
            for (int w = 0; w < 4; ++w) ct[w] = make_uint2(al[w], ah[w]);
            uint2 *sg = reinterpret_cast<uint2 *>(slot + C::SL_SIG);
#pragma unroll
            for (int w = 0; w < 4; ++w) sg[w] = ct[w];
            sample_in_ball<PM::TAU, 32>(ct, blkw, mask);
            uint4 *mo = reinterpret_cast<uint4 *>(slot + C::SL_CM);
#pragma unroll
            for (int k = 0; k < 4; ++k)
                mo[k] = make_uint4(mask[(4 * k) * 32], mask[(4 * k + 1) * 32], mask[(4 * k + 2) * 32], mask[(4 * k + 3) * 32]);
        }
        __threadfence_block();
        __syncwarp();
        if (act) {
            if (drop)
                retire(s, item);
            else
                publish(s, AS_REJ);
        }
        __syncwarp();
    };

    // bounds-checked build: a slot whose item or key index is out of range is dropped (warp-uniform)
    auto bad_slot = [&](unsigned s, unsigned item) -> bool {
        if (!bc_ok(item < n, BC_SIGN_SLOT)) {
            if (lane == 0) publish(s, AS_FREE);
            __syncwarp();
            return true;
        }
        if (!bc_ok(arg.key_idx[item] < arg.nkeys, BC_SIGN_KEY)) {
            if (lane == 0) retire(s, item);
            __syncwarp();
            return true;
        }
        return false;
    };

    // ---------------------------------------------------------------- w = A y (warp per attempt)
    auto w_job = [&](unsigned s) {
        const unsigned item = s_item[s], nonce = s_nonce[s];
        if (bad_slot(s, item)) return;
        if (superseded(item, nonce)) {
            if (lane == 0) retire(s, item);
            __syncwarp();
            return;
        }
        uint8_t *slot = slot_ptr(s);
        const uint8_t *row = arg.cache + (size_t)arg.key_idx[item] * arg.cpitch;
        int32_t *yh = reinterpret_cast<int32_t *>(wa);
        g.sm = yh + L * N + half * NTT_SMEM_WORDS;
#pragma unroll 1
        for (int j0 = 0; j0 < L; j0 += 2) {
            const int j = j0 + half;
            if (j < L) {
                int32_t yc[16], x[16];
                unpack_z_contig<MODE>(yc, slot + C::SL_Y + (size_t)j * PM::POLYZ_PACKED, g.t);
                contig_to_strided(g, yc, x);
                ntt16_ool(x, g.sm, g.gmask, g.t);
                store16_smem(yh + j * N, x, g.t);
            }
        }
        __syncwarp();
        const int32_t *mat0 = reinterpret_cast<const int32_t *>(row + C::SK_MAT);
#pragma unroll 1
        for (int i0 = 0; i0 < K; i0 += 2) {
            const int i = i0 + half;  // K is even
            int32_t acc[16];
#pragma unroll
            for (int m = 0; m < 16; ++m) acc[m] = 0;
#pragma unroll 1
            for (int j0 = 0; j0 < L; j0 += 4) {
                int32_t av[4][16];
#pragma unroll
                for (int jj = 0; jj < 4; ++jj)
                    if (j0 + jj < L) load16_contig(av[jj], mat0 + ((size_t)i * L + j0 + jj) * N + 16 * g.t);
#pragma unroll
                for (int jj = 0; jj < 4; ++jj) {
                    if (j0 + jj < L) {
                        int32_t yv[16];
                        load16_smem(yv, yh + (j0 + jj) * N, g.t);
#pragma unroll
                        for (int m = 0; m < 16; ++m) acc[m] += montmul(av[jj][m], yv[m]);
                    }
                }
            }
#pragma unroll
            for (int m = 0; m < 16; ++m) acc[m] = reduce32(acc[m]);
            intt16_ool(acc, g.sm, g.gmask, g.t);
            // w0 and w1 bytes thread-major (thread t's strided coefficients t + 16 m contiguous)
            int4 *w0t = reinterpret_cast<int4 *>(slot + C::SL_W0 + (size_t)i * C::POLY) + 4 * g.t;
            int32_t w1[16], a0[16];
#pragma unroll
            for (int m = 0; m < 16; ++m) w1[m] = decompose<MODE>(a0[m], caddq(acc[m]));
#pragma unroll
            for (int k = 0; k < 4; ++k) w0t[k] = make_int4(a0[4 * k], a0[4 * k + 1], a0[4 * k + 2], a0[4 * k + 3]);
            {
                uint32_t b[4] = {0u, 0u, 0u, 0u};
#pragma unroll
                for (int m = 0; m < 16; ++m) b[m >> 2] |= ((uint32_t)w1[m] & 0xFFu) << (8 * (m & 3));
                *reinterpret_cast<uint4 *>(slot + C::SL_W1B + (size_t)i * 256 + 16 * g.t) = make_uint4(b[0], b[1], b[2], b[3]);
            }
            int32_t w1c[16];
            strided_to_contig(g, w1, w1c);
            uint32_t v[16];
#pragma unroll
            for (int m = 0; m < 16; ++m) v[m] = (uint32_t)w1c[m];
            pack16_words<PM::W1_BITS>(
                reinterpret_cast<uint32_t *>(slot + C::SL_W1P + (size_t)i * PM::POLYW1_PACKED + g.t * 2 * PM::W1_BITS), v);
        }
        __threadfence_block();
        __syncwarp();
        if (lane == 0) publish(s, AS_CH);
        __syncwarp();
    };

    // ---------------------------------------------------------------- rejection (warp per attempt)
    auto reject_job = [&](unsigned s) {
        const unsigned item = s_item[s], nonce = s_nonce[s];
        if (bad_slot(s, item)) return;
        if (superseded(item, nonce)) {
            if (lane == 0) retire(s, item);
            __syncwarp();
            return;
        }
        uint8_t *slot = slot_ptr(s);
        const uint8_t *row = arg.cache + (size_t)arg.key_idx[item] * arg.cpitch;
        g.sm = reinterpret_cast<int32_t *>(wa) + L * N + half * NTT_SMEM_WORDS;
        uint32_t masks[16];
        {
            const uint4 *mi = reinterpret_cast<const uint4 *>(slot + C::SL_CM);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint4 v = mi[k];
                masks[4 * k] = v.x;
                masks[4 * k + 1] = v.y;
                masks[4 * k + 2] = v.z;
                masks[4 * k + 3] = v.w;
            }
        }
        // both halves transform c (same data, same instructions: no extra time)
        int32_t ch[16];
        challenge_strided(ch, masks, g.t);
        ntt16_ool(ch, g.sm, g.gmask, g.t);
        const int32_t *s1 = reinterpret_cast<const int32_t *>(row + C::SK_S1);
        const int32_t *s2 = reinterpret_cast<const int32_t *>(row + C::SK_S2);
        const int32_t *t0 = reinterpret_cast<const int32_t *>(row + C::SK_T0);
        uint8_t *hs = slot + C::SL_SIG + PM::SIG_H;
        bool rejected = false;
        int n_intt = 0;
        // Acceptance needs every check to pass, so the checks run most selective first: all
        // r0_i = w0_i - invNTT(c s2_i) (kept in place of w0 for the hints), then the z_j, then
        // ct0_i with the hints.  Pairs of polynomials: i / j = 2p + half (K even).
#pragma unroll 1
        for (int i0 = 0; i0 < K && !rejected; i0 += 2) {
            const int i = i0 + half;
            int32_t x[16], r0[16];
            {
                int32_t sv[16];
                load16_contig(sv, s2 + (size_t)i * N + 16 * g.t);
#pragma unroll
                for (int m = 0; m < 16; ++m) x[m] = montmul(ch[m], sv[m]);
            }
            // w0 (thread-major) in flight during the transform
            int32_t *w0t = reinterpret_cast<int32_t *>(slot + C::SL_W0 + (size_t)i * C::POLY) + 16 * g.t;
            load16_contig(r0, w0t);
            intt16_ool(x, g.sm, g.gmask, g.t);
            bool bad = false;
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                r0[m] = reduce32(r0[m] - x[m]);
                bad |= exceeds(r0[m], PM::GAMMA2 - PM::BETA);
            }
            n_intt += 1;
            if (__ballot_sync(FULL, bad)) {
                rejected = true;
                break;
            }
            store16_contig(w0t, r0);
        }
        // z_j = y_j + invNTT(c s1_j)
#pragma unroll 1
        for (int j0 = 0; j0 < L && !rejected; j0 += 2) {
            const int j = j0 + half;
            const bool act = j < L;
            bool bad = false;
            int32_t x[16], y[16];
            if (act) {
                int32_t sv[16];
                load16_contig(sv, s1 + (size_t)j * N + 16 * g.t);
#pragma unroll
                for (int m = 0; m < 16; ++m) x[m] = montmul(ch[m], sv[m]);
                unpack_z_contig<MODE>(y, slot + C::SL_Y + (size_t)j * PM::POLYZ_PACKED, g.t);  // in flight during the transform
            } else {
#pragma unroll
                for (int m = 0; m < 16; ++m) x[m] = y[m] = 0;
            }
            intt16_ool(x, g.sm, g.gmask, g.t);
            n_intt += act ? 1 : 0;
            // z in the contiguous layout of the packing: z[16 t + m] = y + invNTT(c s1)
            int32_t zc[16];
            strided_to_contig(g, x, zc);
            if (act) {
#pragma unroll
                for (int m = 0; m < 16; ++m) {
                    zc[m] = reduce32(zc[m] + y[m]);
                    bad |= exceeds(zc[m], PM::GAMMA1 - PM::BETA);
                }
            }
            if (__ballot_sync(FULL, bad)) {
                rejected = true;
                break;
            }
            if (act) {
                uint32_t v[16];
#pragma unroll
                for (int m = 0; m < 16; ++m) v[m] = (uint32_t)(PM::GAMMA1 - zc[m]);
                pack16_words<PM::Z_BITS>(
                    reinterpret_cast<uint32_t *>(slot + C::SL_SIG + PM::SIG_Z + (size_t)j * PM::POLYZ_PACKED + g.t * 2 * PM::Z_BITS), v);
            }
        }
        // ct0_i = invNTT(c t0_i) and the hints of poly i
        int cnt = 0;
#pragma unroll 1
        for (int i0 = 0; i0 < K && !rejected; i0 += 2) {
            const int i = i0 + half;
            int32_t x[16], r0[16];
            {
                int32_t tv[16];
                load16_contig(tv, t0 + (size_t)i * N + 16 * g.t);
#pragma unroll
                for (int m = 0; m < 16; ++m) x[m] = montmul(ch[m], tv[m]);
            }
            load16_contig(r0, reinterpret_cast<const int32_t *>(slot + C::SL_W0 + (size_t)i * C::POLY) + 16 * g.t);
            const uint4 w1v = *reinterpret_cast<const uint4 *>(slot + C::SL_W1B + (size_t)i * 256 + 16 * g.t);
            intt16_ool(x, g.sm, g.gmask, g.t);
            n_intt += 1;
            bool bad = false;
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                x[m] = reduce32(x[m]);
                bad |= exceeds(x[m], PM::GAMMA2);
            }
            if (__ballot_sync(FULL, bad)) {
                rejected = true;
                break;
            }
            // hint bits of poly i: bit m of hb = hint of coefficient t + 16 m
            const uint32_t w1w[4] = {w1v.x, w1v.y, w1v.z, w1v.w};
            unsigned hb = 0;
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                const int32_t w1 = (int32_t)((w1w[m >> 2] >> (8 * (m & 3))) & 0xFFu);
                hb |= make_hint<MODE>(r0[m] + x[m], w1) << m;
            }
            // counts of both polys of the pair, then positions in ascending coefficient order
            const int mine = __popc(hb);
            int tot = mine;
#pragma unroll
            for (int o = 8; o >= 1; o >>= 1) tot += __shfl_xor_sync(FULL, tot, o);  // sum over the group
            const int tot0 = __shfl_sync(FULL, tot, 0), tot1 = __shfl_sync(FULL, tot, 16);
            if (cnt + tot0 + tot1 > OMEGA) {
                rejected = true;
                break;
            }
            int idx = cnt + (half ? tot0 : 0);
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                const unsigned bit = (hb >> m) & 1u;
                const unsigned bal = (__ballot_sync(FULL, bit) >> lane_off) & 0xFFFFu;
                if (bit) hs[idx + __popc(bal & ((1u << g.t) - 1u))] = (uint8_t)(g.t + 16 * m);
                idx += __popc(bal);
            }
            if (g.t == 0) hs[OMEGA + i] = (uint8_t)(cnt + (half ? tot0 + tot1 : tot0));
            cnt += tot0 + tot1;
        }
        if (g.t == 0) atomicAdd(&s_ctl[CT_INTT], (unsigned)n_intt);  // both halves
        if (rejected) {
            __syncwarp();
            if (lane == 0) retire(s, item);
            __syncwarp();
            return;
        }
        for (int qq = cnt + lane; qq < OMEGA; qq += 32) hs[qq] = 0;
        __threadfence();
        __syncwarp();
        // accepted: lower the item's best nonce; publish if this attempt holds the minimum
        unsigned old = 0;
        if (lane == 0) old = atomicMin(arg.best + item, nonce);
        old = __shfl_sync(FULL, old, 0);
        if (nonce < old) {
            if (lane == 0 && old == 0xFFFFFFFFu) {
                atomicAdd(&q->done_items, 1u);
                atomicSub(&s_ctl[CT_PEND], 1u);
            }
            int got = 0;
            if (lane == 0) {
                for (unsigned spin = 0; spin < arg.lock_spins; ++spin) {
                    if (atomicCAS(arg.locks + item, 0u, 1u) == 0u) {
                        got = 1;
                        break;
                    }
                    __nanosleep(64);
                }
                if (!got) atomicOr(&q->error, 1u);
            }
            got = __shfl_sync(FULL, got, 0);
            if (got) {
                __threadfence();
                unsigned cur = 0;
                if (lane == 0) cur = *reinterpret_cast<volatile unsigned *>(arg.best + item);
                cur = __shfl_sync(FULL, cur, 0);
                if (cur == nonce)
                    publish_signature<PM::SIG_BYTES, 32>(arg.sig_out + (size_t)item * arg.sig_pitch,
                                                         reinterpret_cast<const uint32_t *>(slot + C::SL_SIG), lane);
                __threadfence();
                __syncwarp();
                if (lane == 0) atomicExch(arg.locks + item, 0u);
            }
        }
        __syncwarp();
        if (lane == 0) retire(s, item);
        __syncwarp();
    };

    // ---------------------------------------------------------------- scheduler loop
    long long t_start = clock64();
    unsigned idle = 0, jobs = 0;
    unsigned long long jc[6] = {0, 0, 0, 0, 0, 0};  // cycles: reject, w, challenge, mask, claim, idle
    unsigned jn[6] = {0, 0, 0, 0, 0, 0};
    // a claim that issued nothing is retried only once a slot was freed or the pending count moved
    unsigned no_claim_free = 0xFFFFFFFFu, no_claim_pend = 0xFFFFFFFFu;
#pragma unroll 1
    for (;;) {
        // census of the slot states (each lane looks at NS / 32 slots)
        unsigned cF = 0, cM = 0, cW = 0, cC = 0, cR = 0;
#pragma unroll
        for (int base = 0; base < NS; base += 32) {
            const unsigned st = *reinterpret_cast<volatile unsigned *>(&s_state[base + lane]);
            cF += __popc(__ballot_sync(FULL, st == AS_FREE));
            cM += __popc(__ballot_sync(FULL, st == AS_MASK));
            cW += __popc(__ballot_sync(FULL, st == AS_W));
            cC += __popc(__ballot_sync(FULL, st == AS_CH));
            cR += __popc(__ballot_sync(FULL, st == AS_REJ));
        }
        unsigned pend = *reinterpret_cast<volatile unsigned *>(&s_ctl[CT_PEND]);
        unsigned err = *reinterpret_cast<volatile unsigned *>(&s_ctl[CT_ERR]);
        pend = __shfl_sync(FULL, pend, 0);
        err = __shfl_sync(FULL, err, 0);
        if (err) break;
        if (pend == 0 && cF == (unsigned)NS) break;  // every owned item has its winner, nothing in flight
        const bool other = cR || cC || cW || cM;
        const bool claimable = pend && cF && (cF != no_claim_free || pend != no_claim_pend);
        if (claimable && (cF >= (unsigned)NS / 4 || !other)) {
            unsigned lk = 0;
            if (lane == 0) lk = atomicCAS(&s_ctl[CT_LOCK], 0u, 1u);
            lk = __shfl_sync(FULL, lk, 0);
            if (lk == 0u) {
                const long long tc = clock64();
                const unsigned issued = claim();
                jc[4] += (unsigned long long)(clock64() - tc);
                ++jn[4];
                __threadfence_block();
                if (lane == 0) atomicExch(&s_ctl[CT_LOCK], 0u);
                __syncwarp();
                if (issued) {
                    no_claim_free = no_claim_pend = 0xFFFFFFFFu;
                    idle = 0;
                    continue;
                }
                no_claim_free = cF;
                no_claim_pend = pend;
            }
        }
        // job choice (warp-uniform inputs).  The block keeps one preferred job type, so that at
        // any time most warps run the same code (a small instruction working set, as in a phased
        // kernel) without ever waiting for each other: a warp takes the preferred type while it has
        // a full job's worth of ready slots; otherwise it moves the preference to the type with the
        // most ready work (finishing attempts first on ties) and takes that.
        int job = 0;  // 1 reject, 2 challenge, 3 w, 4 mask
        {
            const unsigned pref = *reinterpret_cast<volatile unsigned *>(&s_ctl[CT_PREF]);
            auto full = [&](int t) {
                return t == 1 ? cR > 0u : t == 2 ? cC >= 32u : t == 3 ? cW > 0u : cM >= (unsigned)MS;
            };
            // ready work in warp jobs: one per reject / w slot, per 32 challenge or MS mask slots
            const unsigned wR = cR, wC = (cC + 31u) / 32u, wW = cW, wM = (cM + MS - 1u) / (unsigned)MS;
            if (pref >= 1u && pref <= 4u && full((int)pref)) {
                job = (int)pref;
            } else {
                unsigned best = 0;
                if (wR > best) { best = wR; job = 1; }
                if (wW > best) { best = wW; job = 3; }
                if (wC > best) { best = wC; job = 2; }
                if (wM > best) { best = wM; job = 4; }
                if (job && lane == 0) atomicExch(&s_ctl[CT_PREF], (unsigned)job);
            }
        }
        const unsigned want_state = job == 1 ? AS_REJ : job == 2 ? AS_CH : job == 3 ? AS_W : AS_MASK;
        const int want = (job == 2) ? 32 : (job == 4 ? MS : 1);
        // take up to `want` slots in that state (lanes race other warps with atomicCAS); the taken
        // slots end up in lanes 0 .. ntaken-1
        unsigned my_slot = 0xFFFFFFFFu;
        int ntaken = 0;
        if (job) {
#pragma unroll 1
            for (int base = 0; base < NS && ntaken < want; base += 32) {
                const unsigned sidx = (unsigned)(base + lane);
                const bool cand = *reinterpret_cast<volatile unsigned *>(&s_state[sidx]) == want_state;
                const unsigned cb = __ballot_sync(FULL, cand);
                const int rank = __popc(cb & ((1u << lane) - 1u));
                bool got = false;
                if (cand && ntaken + rank < want) got = atomicCAS(&s_state[sidx], want_state, AS_BUSY) == want_state;
                const unsigned gb = __ballot_sync(FULL, got);
#pragma unroll 1
                for (unsigned bits = gb; bits; bits &= bits - 1u) {
                    const int src = __ffs(bits) - 1;
                    const unsigned v = __shfl_sync(FULL, sidx, src);
                    if (lane == ntaken + __popc(gb & ((1u << src) - 1u))) my_slot = v;
                }
                ntaken += __popc(gb);
            }
        }
        if (ntaken == 0) {
            if (++idle > arg.idle_polls) {
                if (lane == 0) {
                    atomicOr(&q->error, 4u);
                    atomicExch(&s_ctl[CT_ERR], 1u);
                }
                break;
            }
            const long long ti = clock64();
            __nanosleep(256);
            jc[5] += (unsigned long long)(clock64() - ti);
            ++jn[5];
            continue;
        }
        __threadfence_block();  // the slot data written before its state change is visible from here
        idle = 0;
        ++jobs;
        const long long tj = clock64();
        if (job == 1) {
            reject_job(__shfl_sync(FULL, my_slot, 0));
        } else if (job == 3) {
            w_job(__shfl_sync(FULL, my_slot, 0));
        } else if (job == 2) {
            challenge_job(my_slot, lane < ntaken);
        } else {
            unsigned sl[MS];
#pragma unroll
            for (int a = 0; a < MS; ++a) sl[a] = __shfl_sync(FULL, my_slot, a);
            mask_job(sl, ntaken);
        }
        const int ji = job == 1 ? 0 : job == 3 ? 1 : job == 2 ? 2 : 3;
        jc[ji] += (unsigned long long)(clock64() - tj);
        jn[ji] += (job == 2 || job == 4) ? (unsigned)ntaken : 1u;
    }
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            atomicAdd(&q->jobs[k], jc[k]);
            atomicAdd(&q->jobs[6 + k], (unsigned long long)jn[k]);
        }
    }
    __syncthreads();
    if (tid == 0) {
        atomicAdd(&q->intt, (unsigned long long)s_ctl[CT_INTT]);
        atomicAdd(&q->cyc[3], (unsigned long long)(clock64() - t_start));
    }
    if (lane == 0) atomicAdd(&q->iters, jobs);
}

}  // namespace cudil
