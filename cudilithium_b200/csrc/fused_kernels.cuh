// Fused / persistent form of the batched path (no reference counterpart; the reference drives
// every rejection round from the host, src/api.cu:218-441).
//
//  * Per-key resident cache (built once per key, reused by every message of that key):
//      secret rows  [rho | K | tr | pad..256 | A_hat (K*L polys) | s1_hat | s2_hat | t0_hat]
//      public rows  [rho | tr | pad..256 | A_hat (K*L polys) | t1_hat = NTT(t1 * 2^d)]
//  * k_fused_prehash  one thread per message, longest messages first: mu = H(tr||m), rho' = H(K||mu)
//  * k_fused_sign     ONE persistent kernel for all signing attempts of a batch.  Block b owns the
//                     items b, b + grid, ...; every item has a next-nonce counter, so its nonces are
//                     issued in increasing order, and attempts whose item already has an accepted
//                     smaller nonce are skipped.  Each block claims up to A attempts of its pending
//                     items at a time (speculating more deeply as they run out) and runs them in two
//                     phases per iteration: a Keccak phase (ExpandMask, thread per (attempt, j)
//                     stream; the challenge, thread per attempt) and an NTT phase (w = A*y, 16-thread
//                     group per attempt; rejection checks + hints, warp per attempt).  An accepted
//                     attempt lowers the item's best nonce with atomicMin and, under a per-item lock
//                     with a bounded spin, publishes its signature only if it still holds the
//                     minimum -- the same smallest-accepted-nonce result as deterministic signing
//                     (src/api.cu:388-411).  k_fused_sign_async (fused_sign_async.cuh) runs the same
//                     queue without block-wide phases.
//  * k_fused_verify   persistent verification against public rows (no ExpandA / H(pk) per signature).
#pragma once

#include "keypair_kernels.cuh"
#include "verify_kernels.cuh"

namespace cudil {

template <int MODE>
struct Cache {
    using PM = P<MODE>;
    static constexpr int K = PM::K, L = PM::L;
    static constexpr size_t POLY = N * sizeof(int32_t);
    // secret-key rows
    static constexpr size_t SK_RHO = 0, SK_KEY = 32, SK_TR = 64;
    static constexpr size_t SK_MAT = 256;
    static constexpr size_t SK_S1 = SK_MAT + (size_t)K * L * POLY;
    static constexpr size_t SK_S2 = SK_S1 + (size_t)L * POLY;
    static constexpr size_t SK_T0 = SK_S2 + (size_t)K * POLY;
    static constexpr size_t SK_ROW = SK_T0 + (size_t)K * POLY;
    // public-key rows
    static constexpr size_t PK_RHO = 0, PK_TR = 32;
    static constexpr size_t PK_MAT = 256;
    static constexpr size_t PK_T1 = PK_MAT + (size_t)K * L * POLY;
    static constexpr size_t PK_ROW = PK_T1 + (size_t)K * POLY;
    // per-message prologue output: mu | rho'
    static constexpr size_t ITEM_BYTES = 128;
    // per-attempt slot of the persistent signer
    static constexpr size_t SL_Y = 0;
    static constexpr size_t SL_W0 = align256((size_t)L * PM::POLYZ_PACKED);
    static constexpr size_t SL_W1P = SL_W0 + (size_t)K * POLY;
    static constexpr size_t SL_CM = SL_W1P + align256(PM::W1PACKED_BYTES);
    static constexpr size_t SL_SIG = SL_CM + 256;
    // w1 as bytes, thread-major (byte 16 t + m = coefficient t + 16 m), for the hint computation
    static constexpr size_t SL_W1B = SL_SIG + align256(PM::SIG_BYTES);
    static constexpr size_t SLOT = SL_W1B + (size_t)K * 256;
    // per-signature slot of the persistent verifier: mu | w1' | c masks | status
    static constexpr size_t VS_MU = 0;
    static constexpr size_t VS_W1 = 64;
    static constexpr size_t VS_CM = align256(64 + PM::W1PACKED_BYTES);
    static constexpr size_t VS_STATUS = VS_CM + 64;
    static constexpr size_t VSLOT = VS_CM + 256;
};

// Queue / status block shared by the engine kernels (one per engine, device memory).
struct FusedQueue {
    unsigned long long next_ticket;
    unsigned int done_items;
    // bit 0: a bounded publication-lock wait gave up; bit 1: an item reached its nonce limit (with no
    // accepted nonce its signature row is not written); bit 2: an asynchronous signer block gave up
    // after its idle-poll limit
    unsigned int error;
    unsigned long long attempts;
    unsigned int n;            // items in the current batch
    unsigned int pad;
    unsigned long long intt;   // inverse NTTs run by the rejection checks (for work accounting)
    unsigned int iters;        // signer block-iterations (summed over blocks)
    unsigned int pad2;
    unsigned long long cyc[4]; // signer cycles per phase summed over blocks: claim, keccak, ntt, total
    // asynchronous signer, summed over warps: cycles in reject / w / challenge / ExpandMask / claim /
    // idle polls, then the number of each
    unsigned long long jobs[12];
    // seeded randomized signing (set per batch by the host): rho' of item i is
    // SHAKE256(rho_seed || le64(rho_counter + i), 64); rho_seeded = 0 keeps the other rho' sources
    unsigned long long rho_counter;
    unsigned rho_seeded;
    unsigned pad3;
    uint32_t rho_seed[8];
};

// ------------------------------------------------------------------ cache builders

// Secret rows from packed secret keys (dense, SK_BYTES each): rho, K, tr copied; s1, s2, t0
// unpacked and transformed.  One group per polynomial (+ group p == L+2K copies the seeds).
template <int MODE>
__global__ void __launch_bounds__(kBlock) k_cache_sk(const uint8_t *sk, uint8_t *rows, size_t pitch, int n) {
    using PM = P<MODE>;
    using C = Cache<MODE>;
    constexpr int K = PM::K, L = PM::L, NP = L + 2 * K + 1;
    __shared__ int32_t sm[kGroupsPerBlock * NTT_SMEM_WORDS];
    const int gid = (blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    const int it = gid / NP, p = gid % NP;
    if (it >= n) return;
    Group g = make_group(sm, threadIdx.x >> 4);
    const uint8_t *s = sk + (size_t)it * PM::SK_BYTES;
    uint8_t *row = rows + (size_t)it * pitch;
    if (p == NP - 1) {
        // rho | K | tr are the first 96 bytes of sk
        for (int b = g.t; b < 96; b += 16) row[b] = s[b];
        return;
    }
    int32_t x[16];
    size_t dst;
    if (p < L + K) {
        const uint8_t *src = s + PM::SK_S1 + (size_t)p * PM::POLYETA_PACKED;
#pragma unroll
        for (int i = 0; i < 16; ++i) x[i] = PM::ETA - (int32_t)get_bits(src, (g.t + 16 * i) * PM::ETA_BITS, PM::ETA_BITS);
        dst = (p < L) ? C::SK_S1 + (size_t)p * C::POLY : C::SK_S2 + (size_t)(p - L) * C::POLY;
    } else {
        const uint8_t *src = s + PM::SK_T0 + (size_t)(p - L - K) * POLYT0_PACKED;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            // last coefficient of the last t0 poly ends exactly at SK_BYTES: read 2 bytes only
            const int bit = (g.t + 16 * i) * 13, byte = bit >> 3, sh = bit & 7;
            const uint32_t v = ((uint32_t)src[byte] | ((uint32_t)src[byte + 1] << 8) |
                                (sh + 13 > 16 ? (uint32_t)src[byte + 2] << 16 : 0u)) >> sh;
            x[i] = (1 << (D - 1)) - (int32_t)(v & 0x1FFFu);
        }
        dst = C::SK_T0 + (size_t)(p - L - K) * C::POLY;
    }
    ntt16s(x, g.sm, g.gmask, g.t);
    store16_contig(reinterpret_cast<int32_t *>(row + dst) + 16 * g.t, x);
}

// Public rows: tr = H(pk) and rho (thread per key) ...
template <int MODE>
__global__ void __launch_bounds__(kBlock) k_cache_pk_tr(const uint8_t *pk, uint8_t *rows, size_t pitch, int n) {
    using PM = P<MODE>;
    using C = Cache<MODE>;
    const int it = blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= n) return;
    const uint8_t *p = pk + (size_t)it * PM::PK_BYTES;
    uint8_t *row = rows + (size_t)it * pitch;
    uint32_t al[25], ah[25];
    // pk rows of a dense array are only 4-byte aligned when PK_BYTES % 8 != 0: read bytewise
    struct Src {
        const uint8_t *p;
        __device__ uint2 lane(long long g) const { return load_lane_bytes(p + g * 8, (int)(PM::PK_BYTES - g * 8)); }
    } src{p};
    shake_absorb_prefetch<SHAKE256_RATE>(al, ah, src, PM::PK_BYTES);
    keccak_f1600(al, ah);
    uint2 *tr = reinterpret_cast<uint2 *>(row + C::PK_TR);
#pragma unroll
    for (int w = 0; w < 4; ++w) tr[w] = make_uint2(al[w], ah[w]);
    for (int b = 0; b < 32; ++b) row[C::PK_RHO + b] = p[b];
}

// ... and t1_hat = NTT(t1 * 2^d) (group per polynomial).
template <int MODE>
__global__ void __launch_bounds__(kBlock) k_cache_pk_t1(const uint8_t *pk, uint8_t *rows, size_t pitch, int n) {
    using PM = P<MODE>;
    using C = Cache<MODE>;
    constexpr int K = PM::K;
    __shared__ int32_t sm[kGroupsPerBlock * NTT_SMEM_WORDS];
    const int gid = (blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    const int it = gid / K, i = gid % K;
    if (it >= n) return;
    Group g = make_group(sm, threadIdx.x >> 4);
    const uint8_t *t1p = pk + (size_t)it * PM::PK_BYTES + SEEDBYTES + (size_t)i * POLYT1_PACKED;
    int32_t x[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const int bit = (g.t + 16 * m) * 10, byte = bit >> 3, sh = bit & 7;
        const uint32_t v = ((uint32_t)t1p[byte] | ((uint32_t)t1p[byte + 1] << 8)) >> sh;  // sh + 10 <= 16
        x[m] = (int32_t)((v & 0x3FFu) << D);
    }
    ntt16s(x, g.sm, g.gmask, g.t);
    store16_contig(reinterpret_cast<int32_t *>(rows + (size_t)it * pitch + C::PK_T1 + (size_t)i * C::POLY) + 16 * g.t, x);
}

// ------------------------------------------------------------------ per-batch prologue

// Messages live in one device buffer at 8-byte aligned offsets.  order[] lists the items longest
// first so a warp's messages have similar lengths.
struct MsgRefs {
    const uint8_t *msgs;
    const unsigned long long *offsets;
    const unsigned int *mlens;
    const unsigned int *key_idx;
    const unsigned int *order;
    const uint8_t *rhoprime;  // randomized signing: 64 bytes per item (dense); nullptr = SHAKE256(K || mu)
    unsigned nkeys;           // key-cache rows allocated (bound of key_idx[])
};

// One warp per block, so that the warps holding the longest messages (the order is longest first)
// spread over all SMs.
constexpr int kPrehashBlock = 32;

template <int MODE>
__global__ void __launch_bounds__(kPrehashBlock) k_fused_prehash(const uint8_t *cache, size_t cpitch, MsgRefs mr,
                                                                 uint8_t *items, const FusedQueue *q) {
    using C = Cache<MODE>;
    const unsigned n = q->n;
    for (unsigned r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const unsigned it = mr.order[r];
        if (!bc_ok(it < n && mr.key_idx[it] < mr.nkeys, BC_PREHASH_ITEM)) continue;
        const uint8_t *row = cache + (size_t)mr.key_idx[it] * cpitch;
        uint32_t al[25], ah[25];
        TwoPart src{row + C::SK_TR, 4, mr.msgs + mr.offsets[it], (long long)mr.mlens[it]};
        shake_absorb_prefetch<SHAKE256_RATE>(al, ah, src, (long long)SEEDBYTES + mr.mlens[it]);
        keccak_f1600(al, ah);
        uint2 mu[8];
#pragma unroll
        for (int w = 0; w < 8; ++w) mu[w] = make_uint2(al[w], ah[w]);
        uint2 *out = reinterpret_cast<uint2 *>(items + (size_t)it * C::ITEM_BYTES);
#pragma unroll
        for (int w = 0; w < 8; ++w) out[w] = mu[w];
        if (q->rho_seeded) {
            uint32_t seed[8];
#pragma unroll
            for (int w = 0; w < 8; ++w) seed[w] = q->rho_seed[w];
            uint2 rp[8];
            derive_rhoprime(rp, seed, q->rho_counter + it);
#pragma unroll
            for (int w = 0; w < 8; ++w) out[8 + w] = rp[w];
            continue;
        }
        if (mr.rhoprime) {
            const uint8_t *rp = mr.rhoprime + (size_t)it * CRHBYTES;
#pragma unroll 1
            for (int b = 0; b < CRHBYTES; ++b) items[(size_t)it * C::ITEM_BYTES + 64 + b] = rp[b];
            continue;
        }
        uint2 key[4];
        ld_lanes(key, row + C::SK_KEY);
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
#pragma unroll
        for (int w = 0; w < 8; ++w) out[8 + w] = make_uint2(al[w], ah[w]);
    }
}

// Resets the queue and, for signing, the per-item winner state of q->n items (n set by the host
// copy; best == nullptr: queue only).
static __global__ void k_fused_init(FusedQueue *q, unsigned *best, unsigned *locks, unsigned *next_nonce,
                                    unsigned *inflight) {
    const unsigned n = q->n;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; best && i < n; i += gridDim.x * blockDim.x) {
        best[i] = 0xFFFFFFFFu;
        locks[i] = 0u;
        if (next_nonce) next_nonce[i] = 0u;
        if (inflight) inflight[i] = 0u;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        q->next_ticket = 0;
        q->done_items = 0;
        q->error = 0;
        q->attempts = 0;
        q->intt = 0;
        q->iters = 0;
        for (int i = 0; i < 4; ++i) q->cyc[i] = 0;
        for (int i = 0; i < 12; ++i) q->jobs[i] = 0;
    }
}

// ------------------------------------------------------------------ persistent signer
//
// Work queue.  Block b owns the items b, b + grid, b + 2*grid, ... and schedules them itself, so
// refilling slots touches no shared counter.  Every owned item has a next-nonce counter and an
// in-flight counter; a claim gives pending items (no accepted nonce yet) their next nonce, at most
// D in flight per item, D = spec_slots / pending (1..64).  While a block owning many items has many
// pending, D = 1 and each batch takes half of them, so the two batches in flight hold different
// items and no attempt is wasted (blocks owning fewer than A / 4 items keep D >= 2 so both
// batches stay fed); as pending items run out D grows up to 64, so the last items of a block are
// speculated deeply instead of taking one rejection round after another.
// Nonces of an item are issued in increasing order and every issued attempt completes before the
// block exits, so the winner -- the smallest accepted nonce -- is the deterministic signature.
//
struct FusedSignArgs {
    const uint8_t *cache;
    size_t cpitch;
    const unsigned *key_idx;
    const uint8_t *items;
    uint8_t *sig_out;
    size_t sig_pitch;
    uint8_t *scratch;
    FusedQueue *q;
    unsigned *best, *locks, *next_nonce, *inflight;
    unsigned spec_slots;  // per-block target of attempts in flight (<= 2 * THREADS)
    // bounds of the device-side loops (run-time so that a host can shorten them):
    unsigned nonce_limit;  // nonces an item may use (the 16-bit nonce field allows 65536)
    unsigned lock_spins;   // tries for a per-item publication lock before giving up (error bit 0)
    unsigned idle_polls;   // empty polls before an asynchronous signer block gives up (error bit 2)
    unsigned nkeys;        // key-cache rows allocated (bound of key_idx[])
};

// Sentinel best nonce of an item that used all its nonces without an accepted attempt: below the
// "pending" value 0xFFFFFFFF, above every real nonce, so the item counts as finished (error bit 1).
constexpr unsigned kNonceExhausted = 0xFFFFFFFEu;

template <int MODE, int THREADS>
struct FusedSignSmem {
    using PM = P<MODE>;
    static constexpr int G = THREADS / 16;
    static constexpr size_t CTRL = 4 * THREADS * sizeof(unsigned) + 256;
    static constexpr size_t PH_N = (size_t)G * (PM::L * N * 4 + NTT_SMEM_WORDS * 4);
    static constexpr size_t PH_K = (size_t)THREADS * (34 + 16) * 4;
    static constexpr size_t BYTES = CTRL + (PH_N > PH_K ? PH_N : PH_K);
};

// default bounds of the signer's loops (FusedSignArgs)
constexpr unsigned kNonceLimit = 1u << 16;
constexpr unsigned kLockSpinLimit = 1u << 22;  // x ~64 ns sleeps

// Copies a staged signature (256-byte aligned words) to its output row with NT cooperating
// threads (t = 0 .. NT-1): whole 32-bit words when the row is 4-byte aligned -- full-width writes,
// which matters when the output is pinned host memory written over PCIe -- and bytes otherwise
// and for a last partial word.  Eight words per thread are loaded before they are stored.
template <int BYTES, int NT>
__device__ __forceinline__ void publish_signature(uint8_t *dst, const uint32_t *src, int t) {
    constexpr int NW = (BYTES + 3) / 4, NFULL = BYTES / 4;
    if ((reinterpret_cast<uintptr_t>(dst) & 3u) == 0u) {
        uint32_t *d = reinterpret_cast<uint32_t *>(dst);
#pragma unroll 1
        for (int w0 = 0; w0 < NFULL; w0 += 8 * NT) {
            uint32_t w[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int wi = w0 + t + NT * k;
                w[k] = (wi < NFULL) ? src[wi] : 0u;
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int wi = w0 + t + NT * k;
                if (wi < NFULL) d[wi] = w[k];
            }
        }
        if (NFULL < NW && t < BYTES - 4 * NFULL) dst[4 * NFULL + t] = (uint8_t)(src[NFULL] >> (8 * t));
        return;
    }
#pragma unroll 1
    for (int w0 = 0; w0 < NW; w0 += 8 * NT) {
        uint32_t w[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int wi = w0 + t + NT * k;
            w[k] = (wi < NW) ? src[wi] : 0u;
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int wi = w0 + t + NT * k;
#pragma unroll
            for (int b = 0; b < 4; ++b)
                if (wi < NW && 4 * wi + b < BYTES) dst[4 * wi + b] = (uint8_t)(w[k] >> (8 * b));
        }
    }
}

template <int MODE, int THREADS>
__global__ void __launch_bounds__(THREADS, 512 / THREADS) k_fused_sign(FusedSignArgs arg) {
    using PM = P<MODE>;
    using C = Cache<MODE>;
    constexpr int K = PM::K, L = PM::L, OMEGA = PM::OMEGA, A = THREADS;
    enum { CT_PEND = 0, CT_KJOB, CT_NJOB, CT_NA0, CT_NA1 };
    extern __shared__ __align__(16) uint8_t fs_smem[];
    unsigned *s_item = reinterpret_cast<unsigned *>(fs_smem);   // [2][A]
    unsigned *s_nonce = s_item + 2 * A;                          // [2][A]
    unsigned *s_ctl = s_nonce + 2 * A;                           // CT_* and per-warp counts
    uint8_t *ph = fs_smem + FusedSignSmem<MODE, THREADS>::CTRL;
    FusedQueue *q = arg.q;
    const int tid = threadIdx.x, gi = tid >> 4, lane = tid & 31, lane_off = lane & 16;
    const unsigned n = q->n;
    uint8_t *my_slots = arg.scratch + (size_t)blockIdx.x * 2 * A * C::SLOT;
    auto slot_of = [&](int buf, int a) { return my_slots + ((size_t)buf * A + a) * C::SLOT; };

    Group g;
    g.t = tid & 15;
    g.gmask = 0xFFFFu << lane_off;
    // Dilithium2's signer holds the inlined transforms in its register budget without spilling, so
    // loads issued before a transform overlap it; the larger parameter sets call the out-of-line
    // copies, which keep register use and code size down.
    auto fwd = [&](int32_t (&x)[16]) {
        if constexpr (MODE == 2)
            ntt16s(x, g.sm, g.gmask, g.t);
        else
            ntt16_ool(x, g.sm, g.gmask, g.t);
    };
    auto inv = [&](int32_t (&x)[16]) {
        if constexpr (MODE == 2)
            intt16s(x, g.sm, g.gmask, g.t);
        else
            intt16_ool(x, g.sm, g.gmask, g.t);
    };

    // ---------------- claim: fill batch `buf` with up to A attempts of this block's items
    // (block-collective; warp 0 scans the owned items, one item per lane per pass)
    const unsigned grid = gridDim.x, b0 = blockIdx.x;
    const unsigned n_own = (b0 < n) ? (n - b0 + grid - 1) / grid : 0u;
    auto claim = [&](int buf) {
        if (tid < 32) {
            const unsigned pend = s_ctl[CT_PEND];
            unsigned D = 0;
            if (pend) {
                // depth 1 (alternating halves) needs enough owned items to fill both batches
                const unsigned dmin = (n_own >= (unsigned)A / 4u) ? 1u : 2u;
                const unsigned t = arg.spec_slots / pend;
                D = t < dmin ? dmin : (t > 64u ? 64u : t);
            }
            // With one attempt per item (D == 1) a batch takes at most half of the pending items, so
            // the two batches in flight hold different items and no attempt is speculative.
            const unsigned cap = (D == 1u) ? ((pend + 1u) / 2u < (unsigned)A ? (pend + 1u) / 2u : (unsigned)A) : (unsigned)A;
            unsigned filled = 0;
            // An item with f attempts in flight gets D - f more (none when f >= D).  When all of
            // them fit the batch (D * pend <= cap), one scan hands each item its attempts with one
            // atomic on its nonce counter; otherwise pass p gives one more attempt to the items
            // with at most p in flight, so a full batch spreads its slots over the items.
            const bool one_scan = D >= 2u && D * pend <= cap;
            auto place = [&](unsigned pos, unsigned i, unsigned nn) {
                s_item[buf * A + pos] = i;
                if (nn < arg.nonce_limit) {
                    s_nonce[buf * A + pos] = nn;
                } else {
                    // every nonce used without acceptance (never for honest keys at the default
                    // limit): the slot becomes a no-op, and the first lane to get here marks the
                    // item finished so that the block can exit
                    s_nonce[buf * A + pos] = 0xFFFFFFFFu;
                    if (atomicCAS(arg.best + i, 0xFFFFFFFFu, kNonceExhausted) == 0xFFFFFFFFu) {
                        atomicOr(&q->error, 2u);
                        atomicSub(&s_ctl[CT_PEND], 1u);
                    }
                }
            };
#pragma unroll 1
            for (unsigned k0 = 0; one_scan && k0 < n_own; k0 += 32) {
                const unsigned k = k0 + lane, i = b0 + k * grid;
                unsigned want = 0;
                if (k < n_own) {
                    const unsigned bi = __ldcg(arg.best + i), fi = __ldcg(arg.inflight + i);
                    want = (bi == 0xFFFFFFFFu && fi < D) ? D - fi : 0u;
                }
                unsigned incl = want;  // inclusive prefix sum over the warp
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const unsigned v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                    if (lane >= o) incl += v;
                }
                const unsigned pos0 = filled + incl - want;
                // (D * pend <= cap keeps every position below cap; the clamp only guards the bound)
                const unsigned take = pos0 >= cap ? 0u : (want < cap - pos0 ? want : cap - pos0);
                if (take) {
                    const unsigned nn = atomicAdd(arg.next_nonce + i, take);
                    atomicAdd(arg.inflight + i, take);
#pragma unroll 1
                    for (unsigned r = 0; r < take; ++r) place(pos0 + r, i, nn + r);
                }
                filled += __shfl_sync(0xFFFFFFFFu, incl, 31);
                if (filled > cap) filled = cap;
            }
#pragma unroll 1
            for (unsigned pass = 0; !one_scan && pass < D && filled < cap; ++pass) {
#pragma unroll 1
                for (unsigned k0 = 0; k0 < n_own && filled < cap; k0 += 32) {
                    const unsigned k = k0 + lane, i = b0 + k * grid;
                    bool ok = false;
                    if (k < n_own) {
                        // both loads issued together (one round trip, not two dependent ones)
                        const unsigned bi = __ldcg(arg.best + i), fi = __ldcg(arg.inflight + i);
                        ok = bi == 0xFFFFFFFFu && fi <= pass;
                    }
                    const unsigned bal = __ballot_sync(0xFFFFFFFFu, ok);
                    const unsigned pos = filled + __popc(bal & ((1u << lane) - 1u));
                    if (ok && pos < cap) {
                        const unsigned nn = atomicAdd(arg.next_nonce + i, 1u);
                        atomicAdd(arg.inflight + i, 1u);
                        place(pos, i, nn);
                    }
                    filled += __popc(bal);
                    if (filled > cap) filled = cap;
                }
            }
            if (lane == 0) {
                s_ctl[CT_NA0 + buf] = filled;
                s_ctl[CT_KJOB] = 0;
                s_ctl[CT_NJOB] = 0;
                if (filled) atomicAdd(&q->attempts, (unsigned long long)filled);
            }
        }
        __syncthreads();
    };

    // ---------------- Keccak phase: challenge of batch cb (jobs < na_c), ExpandMask of batch nb
    auto keccak_phase = [&](int cb, int na_c, int nb, int na_n) {
        uint32_t *blkw = reinterpret_cast<uint32_t *>(ph) + tid;
        uint32_t *mask = reinterpret_cast<uint32_t *>(ph) + 34 * THREADS + tid;
        // ExpandMask jobs start at a multiple of 32, so no warp holds both job types (a warp runs
        // divergent branches one after the other: a mixed warp would take 8 + 5 permutations)
        const int cpad = (na_c + 31) & ~31;
        const int total = cpad + na_n * L;
        // a warp takes 32 consecutive jobs at a time, so its lanes run the same job type together
#pragma unroll 1
        for (;;) {
            unsigned base = 0;
            if (lane == 0) base = atomicAdd(&s_ctl[CT_KJOB], 32u);
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if ((int)base >= total) break;
            const int job = (int)base + lane;
            // attempts above an already accepted nonce of their item are skipped (they cannot win)
            if (job < na_c) {
                const unsigned item = bc_ok(job < A, BC_SIGN_SLOT) ? s_item[cb * A + job] : 0xFFFFFFFFu;
                if (bc_ok(item < n, BC_SIGN_SLOT) && !(__ldcg(arg.best + item) < s_nonce[cb * A + job])) {
                    uint8_t *slot = slot_of(cb, job);
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
                    sample_in_ball<PM::TAU, THREADS>(ct, blkw, mask);
                    uint4 *mo = reinterpret_cast<uint4 *>(slot + C::SL_CM);
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        mo[k] = make_uint4(mask[(4 * k) * THREADS], mask[(4 * k + 1) * THREADS], mask[(4 * k + 2) * THREADS],
                                           mask[(4 * k + 3) * THREADS]);
                }
            } else if (job >= cpad && job < total) {
                const int idx = job - cpad, a = idx / L, j = idx % L;
                const bool slot_ok = bc_ok(a < A, BC_SIGN_SLOT);
                const unsigned item = slot_ok ? s_item[nb * A + a] : 0xFFFFFFFFu, nonce = slot_ok ? s_nonce[nb * A + a] : 0u;
                if (bc_ok(item < n, BC_SIGN_SLOT) && !(__ldcg(arg.best + item) < nonce)) {
                    uint2 rhop[8];
                    ld_lanes(rhop, arg.items + (size_t)item * C::ITEM_BYTES + 64);
                    expand_mask_stream<MODE>(slot_of(nb, a) + C::SL_Y + (size_t)j * PM::POLYZ_PACKED, rhop,
                                             (uint32_t)(L * nonce + j));
                }
            }
            __syncwarp();  // every lane runs the same grab / sync sequence
        }
    };

    // rejection checks, hints and publication of one attempt (warp-collective).  The two groups
    // of the warp take the attempt's polynomials in pairs (poly 2p + half), so they follow the same
    // control flow: a rejection ends the job for the whole warp, and no group waits for another
    // group's longer attempt.
    auto reject_job = [&](int cb, int a) {
        // (range checks of the bounds-checked build: every value is the same across the warp)
        if (!bc_ok(a < A, BC_SIGN_SLOT)) return;
        const unsigned item = s_item[cb * A + a], nonce = s_nonce[cb * A + a];
        if (!bc_ok(item < n, BC_SIGN_SLOT)) return;
        // one decision per warp: out-of-range nonce, or a smaller nonce of the item already accepted
        bool skip = nonce > 0xFFFFu || __ldcg(arg.best + item) < nonce;
        skip = __shfl_sync(0xFFFFFFFFu, skip, 0);
        const unsigned key = arg.key_idx[item];
        if (skip || !bc_ok(key < arg.nkeys, BC_SIGN_KEY)) {
            if (lane == 0) atomicSub(arg.inflight + item, 1u);
            return;
        }
        uint8_t *slot = slot_of(cb, a);
        const uint8_t *row = arg.cache + (size_t)key * arg.cpitch;
        g.sm = reinterpret_cast<int32_t *>(ph) + (size_t)gi * (L * N + NTT_SMEM_WORDS) + L * N;
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
        // both groups transform c (same data, same instructions)
        int32_t ch[16];
        challenge_strided(ch, masks, g.t);
        fwd(ch);
        const int32_t *s1 = reinterpret_cast<const int32_t *>(row + C::SK_S1);
        const int32_t *s2 = reinterpret_cast<const int32_t *>(row + C::SK_S2);
        const int32_t *t0 = reinterpret_cast<const int32_t *>(row + C::SK_T0);
        uint8_t *hs = slot + C::SL_SIG + PM::SIG_H;
        const int half = lane_off >> 4;
        bool rejected = false;
        int n_intt = 0, cnt = 0;
        // Acceptance needs every check to pass, so the checks run most selective first: pair steps
        // of the r0_i (r0 replaces w0 in the slot, for the hints), then of the z_j, then of the
        // ct0_i with the hints.  K is even for every parameter set; L is odd for two of them, so
        // the last z pair may leave the second group without a polynomial (it transforms zeros
        // and stores nothing).  While one step transforms, the next step's key rows and (inlined
        // transforms) this step's slot data are in flight.
        constexpr int PR = K / 2, PZ = (L + 1) / 2, NSTEP = 2 * PR + PZ;
        auto operand = [&](int step) -> const int32_t * {
            if (step < PR) return s2 + (size_t)(2 * step + half) * N;
            if (step < PR + PZ) {
                const int j = 2 * (step - PR) + half;
                return s1 + (size_t)(j < L ? j : L - 1) * N;
            }
            return t0 + (size_t)(2 * (step - PR - PZ) + half) * N;
        };
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
            int32_t *w0 = reinterpret_cast<int32_t *>(slot + C::SL_W0) + (size_t)(is_z ? 0 : k) * N;
            const uint8_t *yp = slot + C::SL_Y + (size_t)(act ? k : 0) * PM::POLYZ_PACKED;
            int32_t pre[16];
            // the slot data of the step: with the inlined transform it is in flight across it; the
            // out-of-line transform would spill a load held across the call, so there it is read
            // afterwards
            auto load_pre = [&] {
                if (is_z) {
                    unpack_z_strided<MODE>(pre, yp, g.t);
#pragma unroll
                    for (int m = 0; m < 16; ++m) pre[m] = act ? pre[m] : 0;
                } else {
                    load16_strided(pre, w0, g.t);
                }
            };
            if constexpr (MODE == 2) load_pre();
            inv(x);
            n_intt += act ? 1 : 0;
            if constexpr (MODE != 2) load_pre();
            bool bad = false;
            if (is_z) {
#pragma unroll
                for (int m = 0; m < 16; ++m) {
                    x[m] = reduce32(x[m] + pre[m]);
                    bad |= act && exceeds(x[m], PM::GAMMA1 - PM::BETA);
                }
                if (__ballot_sync(0xFFFFFFFFu, bad)) {
                    rejected = true;
                    break;
                }
                int32_t zc[16];
                strided_to_contig(g, x, zc);
                if (act) {
                    uint32_t v[16];
#pragma unroll
                    for (int m = 0; m < 16; ++m) v[m] = (uint32_t)(PM::GAMMA1 - zc[m]);
                    pack16_words<PM::Z_BITS>(
                        reinterpret_cast<uint32_t *>(slot + C::SL_SIG + PM::SIG_Z + (size_t)k * PM::POLYZ_PACKED + g.t * 2 * PM::Z_BITS), v);
                }
            } else if (is_r0) {
#pragma unroll
                for (int m = 0; m < 16; ++m) {
                    pre[m] = reduce32(pre[m] - x[m]);
                    bad |= exceeds(pre[m], PM::GAMMA2 - PM::BETA);
                }
                if (__ballot_sync(0xFFFFFFFFu, bad)) {
                    rejected = true;
                    break;
                }
                store16_strided(w0, pre, g.t);
            } else {
#pragma unroll
                for (int m = 0; m < 16; ++m) {
                    x[m] = reduce32(x[m]);
                    bad |= exceeds(x[m], PM::GAMMA2);
                }
                if (__ballot_sync(0xFFFFFFFFu, bad)) {
                    rejected = true;
                    break;
                }
                // hint bits of poly k: bit m of hb = hint of coefficient t + 16 m
                const uint8_t *w1p = slot + C::SL_W1P + (size_t)k * PM::POLYW1_PACKED;
                unsigned hb = 0;
#pragma unroll
                for (int m = 0; m < 16; ++m) {
                    const int32_t w1 = (int32_t)get_bits(w1p, (g.t + 16 * m) * PM::W1_BITS, PM::W1_BITS);
                    hb |= make_hint<MODE>(pre[m] + x[m], w1) << m;
                }
                // hint counts of both polynomials of the pair (sums over each group), then the
                // positions in ascending coefficient order: poly 2p first, then poly 2p + 1
                int tot = __popc(hb);
#pragma unroll
                for (int o = 8; o >= 1; o >>= 1) tot += __shfl_xor_sync(0xFFFFFFFFu, tot, o);
                const int tot0 = __shfl_sync(0xFFFFFFFFu, tot, 0), tot1 = __shfl_sync(0xFFFFFFFFu, tot, 16);
                if (cnt + tot0 + tot1 > OMEGA) {
                    rejected = true;
                    break;
                }
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
        n_intt += __shfl_down_sync(0xFFFFFFFFu, n_intt, 16);  // lane 0: both groups
        if (lane == 0) {
            atomicAdd(&q->intt, (unsigned long long)n_intt);
            atomicSub(arg.inflight + item, 1u);
        }
        if (rejected) return;
        for (int qq = cnt + lane; qq < OMEGA; qq += 32) hs[qq] = 0;
        __syncwarp();
        // accepted: lower the item's best nonce; publish if this attempt holds the minimum
        unsigned old = 0;
        if (lane == 0) old = atomicMin(arg.best + item, nonce);
        old = __shfl_sync(0xFFFFFFFFu, old, 0);
        if (nonce >= old) return;
        if (lane == 0 && old == 0xFFFFFFFFu) {
            atomicAdd(&q->done_items, 1u);
            atomicSub(&s_ctl[CT_PEND], 1u);
        }
        // (old == kNonceExhausted: the item was already counted as finished; a late acceptance
        // below the limit still publishes its signature)
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
        got = __shfl_sync(0xFFFFFFFFu, got, 0);
        if (!got) return;
        __threadfence();
        unsigned cur = 0;
        if (lane == 0) cur = *reinterpret_cast<volatile unsigned *>(arg.best + item);
        cur = __shfl_sync(0xFFFFFFFFu, cur, 0);
        if (cur == nonce) {
            publish_signature<PM::SIG_BYTES, 32>(arg.sig_out + (size_t)item * arg.sig_pitch,
                                                 reinterpret_cast<const uint32_t *>(slot + C::SL_SIG), lane);
        }
        __threadfence();
        __syncwarp();
        if (lane == 0) atomicExch(arg.locks + item, 0u);
    };

    // w = invNTT(A_hat * NTT(y)), Decompose, pack w1 of one attempt (group-collective)
    auto w_job = [&](int nb, int a) {
        if (!bc_ok(a < A, BC_SIGN_SLOT)) return;
        const unsigned item = s_item[nb * A + a];
        if (!bc_ok(item < n, BC_SIGN_SLOT)) return;
        bool skip = __ldcg(arg.best + item) < s_nonce[nb * A + a];
        skip = __shfl_sync(g.gmask, skip, lane_off);
        const unsigned key = arg.key_idx[item];
        if (skip || !bc_ok(key < arg.nkeys, BC_SIGN_KEY)) return;
        uint8_t *slot = slot_of(nb, a);
        const uint8_t *row = arg.cache + (size_t)key * arg.cpitch;
        int32_t *yh = reinterpret_cast<int32_t *>(ph) + (size_t)gi * (L * N + NTT_SMEM_WORDS);
        g.sm = yh + L * N;
#pragma unroll 1
        for (int j = 0; j < L; ++j) {
            int32_t x[16];
            unpack_z_strided<MODE>(x, slot + C::SL_Y + (size_t)j * PM::POLYZ_PACKED, g.t);
            fwd(x);
            store16_smem(yh + j * N, x, g.t);
        }
        __syncwarp(g.gmask);
        const int32_t *mat0 = reinterpret_cast<const int32_t *>(row + C::SK_MAT);
#pragma unroll 1
        for (int i = 0; i < K; ++i) {
            int32_t acc[16];
#pragma unroll
            for (int m = 0; m < 16; ++m) acc[m] = 0;
            // A row entries in chunks of up to four polynomials: their loads are all in flight
            // before the first one is consumed
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
            inv(acc);
            int32_t *w0 = reinterpret_cast<int32_t *>(slot + C::SL_W0) + (size_t)i * N;
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
            pack16_words<PM::W1_BITS>(
                reinterpret_cast<uint32_t *>(slot + C::SL_W1P + (size_t)i * PM::POLYW1_PACKED + g.t * 2 * PM::W1_BITS), v);
        }
        __syncwarp(g.gmask);
    };

    // ---------------- NTT phase: rejection of batch cb, w = A y of batch nb
    auto ntt_phase = [&](int cb, int na_c, int nb, int na_n) {
        // a warp takes one unit at a time: a rejection unit is one attempt for the whole warp, a w
        // unit two attempts, one per 16-thread group (w jobs have no data-dependent control flow,
        // so the two groups run in lockstep)
        const int total = na_c + (na_n + 1) / 2;
#pragma unroll 1
        for (;;) {
            unsigned base = 0;
            if (lane == 0) base = atomicAdd(&s_ctl[CT_NJOB], 1u);
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if ((int)base >= total) break;
            if ((int)base < na_c) {
                reject_job(cb, (int)base);
            } else {
                const int a = 2 * ((int)base - na_c) + (lane_off ? 1 : 0);
                if (a < na_n) w_job(nb, a);
            }
            __syncwarp();  // both groups back together before the next full-warp grab
        }
    };

    // ---------------- main loop (thread 0 accumulates per-phase cycles for the work counters)
    long long t_claim = 0, t_kec = 0, t_ntt = 0, t_start = clock64(), t0;
    unsigned iters = 0;
    if (tid == 0) s_ctl[CT_PEND] = n_own;
    __syncthreads();
    claim(0);
    keccak_phase(0, 0, 0, (int)s_ctl[CT_NA0]);
    __syncthreads();
    ntt_phase(0, 0, 0, (int)s_ctl[CT_NA0]);
    __syncthreads();
    int cur = 0;
#pragma unroll 1
    for (;;) {
        const int nxt = cur ^ 1;
        t0 = clock64();
        claim(nxt);
        t_claim += clock64() - t0;
        const int na_c = (int)s_ctl[CT_NA0 + cur], na_n = (int)s_ctl[CT_NA0 + nxt];
        // nothing in flight and nothing claimable: every owned item has its winner
        if (na_c == 0 && na_n == 0) break;
        ++iters;
        t0 = clock64();
        keccak_phase(cur, na_c, nxt, na_n);
        __syncthreads();
        t_kec += clock64() - t0;
        t0 = clock64();
        ntt_phase(cur, na_c, nxt, na_n);
        __syncthreads();
        t_ntt += clock64() - t0;
        cur = nxt;
    }
    if (tid == 0) {
        atomicAdd(&q->cyc[0], (unsigned long long)t_claim);
        atomicAdd(&q->cyc[1], (unsigned long long)t_kec);
        atomicAdd(&q->cyc[2], (unsigned long long)t_ntt);
        atomicAdd(&q->cyc[3], (unsigned long long)(clock64() - t_start));
        atomicAdd(&q->iters, iters);
    }
}

// ------------------------------------------------------------------ persistent verifier

// mu = H(tr || m) of every signature of a verification batch, ahead of the persistent verifier
// (as k_fused_prehash for signing): one thread per message, longest first, one warp per block, the
// absorb with the next block's lanes in flight.  A long message therefore costs its own
// permutations on one thread instead of stalling a verifier block's first phase.
template <int MODE>
__global__ void __launch_bounds__(kPrehashBlock) k_fused_verify_prehash(const uint8_t *cache, size_t cpitch, MsgRefs mr,
                                                                        uint8_t *items, const FusedQueue *q) {
    using C = Cache<MODE>;
    const unsigned n = q->n;
    for (unsigned r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const unsigned it = mr.order[r];
        if (!bc_ok(it < n && mr.key_idx[it] < mr.nkeys, BC_PREHASH_ITEM)) continue;
        const uint8_t *row = cache + (size_t)mr.key_idx[it] * cpitch;
        uint32_t al[25], ah[25];
        TwoPart src{row + C::PK_TR, 4, mr.msgs + mr.offsets[it], (long long)mr.mlens[it]};
        shake_absorb_prefetch<SHAKE256_RATE>(al, ah, src, (long long)SEEDBYTES + mr.mlens[it]);
        keccak_f1600(al, ah);
        uint2 *out = reinterpret_cast<uint2 *>(items + (size_t)it * C::ITEM_BYTES);
#pragma unroll
        for (int w = 0; w < 8; ++w) out[w] = make_uint2(al[w], ah[w]);
    }
}

template <int MODE, int THREADS>
struct FusedVerifySmem {
    using PM = P<MODE>;
    static constexpr int G = THREADS / 16;
    static constexpr size_t PH_W = (size_t)G * ((PM::L + 1) * N * 4 + NTT_SMEM_WORDS * 4 + 32);
    static constexpr size_t PH_C = (size_t)THREADS * (34 + 16) * 4;
    static constexpr size_t BYTES = 256 + (PH_W > PH_C ? PH_W : PH_C);
};

template <int MODE, int THREADS>
__global__ void __launch_bounds__(THREADS, 512 / THREADS) k_fused_verify(const uint8_t *cache, size_t cpitch, MsgRefs mr,
                                                          const uint8_t *sig, size_t sig_pitch, int *ret,
                                                          uint8_t *scratch, const uint8_t *items, FusedQueue *q) {
    using PM = P<MODE>;
    using C = Cache<MODE>;
    constexpr int K = PM::K, L = PM::L, OMEGA = PM::OMEGA, A = THREADS, G = THREADS / 16;
    extern __shared__ __align__(16) uint8_t fv_smem[];
    unsigned *s_ctl = reinterpret_cast<unsigned *>(fv_smem);
    uint8_t *ph = fv_smem + 256;
    const int tid = threadIdx.x, gi = tid >> 4, lane = tid & 31;
    const unsigned n = q->n;
    uint8_t *my_slots = scratch + (size_t)blockIdx.x * A * C::VSLOT;
    // chunks of at most A signatures, small enough that every block of the grid gets work
    unsigned chunk = (n + gridDim.x - 1) / gridDim.x;
    chunk = chunk < 1u ? 1u : (chunk > (unsigned)A ? (unsigned)A : chunk);
    for (;;) {
        if (tid == 0) s_ctl[0] = (unsigned)atomicAdd(&q->next_ticket, (unsigned long long)chunk);
        __syncthreads();
        const unsigned base = s_ctl[0];
        if (base >= n) break;
        const int na = (int)((n - base) < chunk ? (n - base) : chunk);

        // hint encoding checks, mu (from the prehash kernel), c = SampleInBall(c~): thread per signature
        if (tid < na) {
            const unsigned it = base + tid;
            const uint8_t *s = sig + (size_t)it * sig_pitch;
            uint8_t *slot = my_slots + (size_t)tid * C::VSLOT;
            int status = bc_ok(mr.key_idx[it] < mr.nkeys, BC_VERIFY_KEY) ? 0 : 4;
            const uint8_t *h = s + PM::SIG_H;
            int k = 0;
            for (int i = 0; i < K && !status; ++i) {
                const int end = h[OMEGA + i];
                if (end < k || end > OMEGA) {
                    status = 1;
                    break;
                }
                for (int j = k + 1; j < end; ++j)
                    if (h[j] <= h[j - 1]) status = 1;
                k = end;
            }
            if (!status)
                for (int j = k; j < OMEGA; ++j)
                    if (h[j]) status = 1;
            uint2 mu8[8];
            ld_lanes(mu8, items + (size_t)it * C::ITEM_BYTES);
            uint2 *mu = reinterpret_cast<uint2 *>(slot + C::VS_MU);
#pragma unroll
            for (int w = 0; w < 8; ++w) mu[w] = mu8[w];
            uint2 ct[4];
#pragma unroll
            for (int w = 0; w < 4; ++w) ct[w] = make_uint2(load_lane_bytes(s + 8 * w, 8).x, load_lane_bytes(s + 8 * w, 8).y);
            uint32_t *blkw = reinterpret_cast<uint32_t *>(ph) + tid;
            uint32_t *mask = reinterpret_cast<uint32_t *>(ph) + 34 * THREADS + tid;
            sample_in_ball<PM::TAU, THREADS>(ct, blkw, mask);
            uint4 *mo = reinterpret_cast<uint4 *>(slot + C::VS_CM);
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)
                mo[kk] = make_uint4(mask[(4 * kk) * THREADS], mask[(4 * kk + 1) * THREADS], mask[(4 * kk + 2) * THREADS],
                                    mask[(4 * kk + 3) * THREADS]);
            reinterpret_cast<int *>(slot + C::VS_STATUS)[0] = status;
        }
        __syncthreads();

        // z norm check + NTT(z), NTT(c), w' = A_hat z_hat - c_hat t1_hat, UseHint, pack: group per signature
        {
            int32_t *zh = reinterpret_cast<int32_t *>(ph) + (size_t)gi * ((L + 1) * N + NTT_SMEM_WORDS + 8);
            uint32_t *hbits = reinterpret_cast<uint32_t *>(zh + (L + 1) * N + NTT_SMEM_WORDS);
            Group g;
            g.t = tid & 15;
            g.gmask = 0xFFFFu << (lane & 16);
            g.sm = zh + (L + 1) * N;
            for (int a = gi; a < na; a += G) {
                const unsigned it = base + a;
                const uint8_t *s = sig + (size_t)it * sig_pitch;
                const unsigned key = mr.key_idx[it];
                const uint8_t *row = cache + (size_t)(bc_ok(key < mr.nkeys, BC_VERIFY_KEY) ? key : 0u) * cpitch;
                uint8_t *slot = my_slots + (size_t)a * C::VSLOT;
                bool zbad = false;
#pragma unroll 1
                for (int j = 0; j < L; ++j) {
                    int32_t x[16];
#pragma unroll
                    for (int m = 0; m < 16; ++m) {
                        const int bit = (g.t + 16 * m) * PM::Z_BITS;
                        const uint8_t *pz = s + PM::SIG_Z + (size_t)j * PM::POLYZ_PACKED + (bit >> 3);
                        const uint32_t v = ((uint32_t)pz[0] | ((uint32_t)pz[1] << 8) | ((uint32_t)pz[2] << 16)) >> (bit & 7);
                        x[m] = PM::GAMMA1 - (int32_t)(v & ((1u << PM::Z_BITS) - 1u));
                        zbad |= exceeds(x[m], PM::GAMMA1 - PM::BETA);
                    }
                    ntt16s(x, g.sm, g.gmask, g.t);
                    store16_smem(zh + j * N, x, g.t);
                }
                if (group_any(g, zbad) && g.t == 0) reinterpret_cast<int *>(slot + C::VS_STATUS)[0] |= 2;
                {
                    uint32_t masks[16];
                    const uint4 *mi = reinterpret_cast<const uint4 *>(slot + C::VS_CM);
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) {
                        const uint4 v = mi[kk];
                        masks[4 * kk] = v.x;
                        masks[4 * kk + 1] = v.y;
                        masks[4 * kk + 2] = v.z;
                        masks[4 * kk + 3] = v.w;
                    }
                    int32_t x[16];
                    challenge_strided(x, masks, g.t);
                    ntt16s(x, g.sm, g.gmask, g.t);
                    store16_smem(zh + L * N, x, g.t);
                }
                __syncwarp(g.gmask);
                const uint8_t *h = s + PM::SIG_H;
#pragma unroll 1
                for (int i = 0; i < K; ++i) {
                    if (g.t < 8) hbits[g.t] = 0;
                    __syncwarp(g.gmask);
                    const int start = (i == 0) ? 0 : h[OMEGA + i - 1];
                    int end = h[OMEGA + i];
                    if (end > OMEGA) end = OMEGA;
                    for (int j = start + g.t; j < end; j += 16) atomicOr(&hbits[h[j] >> 5], 1u << (h[j] & 31));
                    __syncwarp(g.gmask);
                    const int32_t *mat = reinterpret_cast<const int32_t *>(row + C::PK_MAT) + (size_t)i * L * N;
                    int32_t acc[16];
#pragma unroll
                    for (int m = 0; m < 16; ++m) acc[m] = 0;
                    // sum_j A_ij z_j - c t1_i, the key operands in chunks of up to four polynomials
                    // whose loads are all in flight before the first one is consumed (one memory
                    // round trip per chunk).  When L is not a multiple of four, t1_i joins the last
                    // chunk of A row entries as operand L (its shared-memory vector, after
                    // z_hat_0..L-1, is c_hat); otherwise it would start a chunk of its own, and
                    // the separate load below measured faster.  The int32 sum is exact
                    // (|acc| < (L+1) q), so both forms give the same result.
                    const int32_t *t1 = reinterpret_cast<const int32_t *>(row + C::PK_T1) + (size_t)i * N;
                    constexpr int LAST = (L % 4 == 0) ? L - 1 : L;  // last operand in the chunks
#pragma unroll 1
                    for (int j0 = 0; j0 <= LAST; j0 += 4) {
                        int32_t av[4][16];
#pragma unroll
                        for (int jj = 0; jj < 4; ++jj)
                            if (j0 + jj <= LAST) load16_contig(av[jj], (j0 + jj < L ? mat + (size_t)(j0 + jj) * N : t1) + 16 * g.t);
#pragma unroll
                        for (int jj = 0; jj < 4; ++jj) {
                            if (j0 + jj <= LAST) {
                                int32_t zv[16];
                                load16_smem(zv, zh + (j0 + jj) * N, g.t);
                                if (j0 + jj < L) {
#pragma unroll
                                    for (int m = 0; m < 16; ++m) acc[m] += montmul(av[jj][m], zv[m]);
                                } else {
#pragma unroll
                                    for (int m = 0; m < 16; ++m) acc[m] -= montmul(zv[m], av[jj][m]);
                                }
                            }
                        }
                    }
                    if constexpr (LAST < L) {
                        int32_t cv[16], tv[16];
                        load16_smem(cv, zh + L * N, g.t);
                        load16_contig(tv, t1 + 16 * g.t);
#pragma unroll
                        for (int m = 0; m < 16; ++m) acc[m] -= montmul(cv[m], tv[m]);
                    }
#pragma unroll
                    for (int m = 0; m < 16; ++m) acc[m] = reduce32(acc[m]);
                    intt16s(acc, g.sm, g.gmask, g.t);
                    int32_t w1[16];
#pragma unroll
                    for (int m = 0; m < 16; ++m) {
                        const int c = g.t + 16 * m;
                        w1[m] = use_hint<MODE>(caddq(acc[m]), (hbits[c >> 5] >> (c & 31)) & 1u);
                    }
                    int32_t w1c[16];
                    strided_to_contig(g, w1, w1c);
                    uint32_t v[16];
#pragma unroll
                    for (int m = 0; m < 16; ++m) v[m] = (uint32_t)w1c[m];
                    pack16_words<PM::W1_BITS>(
                        reinterpret_cast<uint32_t *>(slot + C::VS_W1 + (size_t)i * PM::POLYW1_PACKED + g.t * 2 * PM::W1_BITS), v);
                    __syncwarp(g.gmask);
                }
            }
        }
        __syncthreads();

        // c~' = H(mu || w1') and compare: thread per signature
        if (tid < na) {
            const unsigned it = base + tid;
            const uint8_t *s = sig + (size_t)it * sig_pitch;
            uint8_t *slot = my_slots + (size_t)tid * C::VSLOT;
            uint32_t al[25], ah[25];
            AlignedBytes src{slot + C::VS_MU, CRHBYTES + PM::W1PACKED_BYTES};
            shake_absorb<SHAKE256_RATE>(al, ah, src, CRHBYTES + PM::W1PACKED_BYTES);
            keccak_f1600(al, ah);
            bool eq = true;
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                const uint2 v = load_lane_bytes(s + 8 * w, 8);
                eq &= (v.x == al[w]) && (v.y == ah[w]);
            }
            const int status = reinterpret_cast<const int *>(slot + C::VS_STATUS)[0];
            ret[it] = (eq && status == 0) ? 0 : -1;
        }
        __syncthreads();
    }
}

}  // namespace cudil
