/*
 * cudilithium_b200 -- C ABI of the B200 batched Dilithium (round 3, v3.1) engine.
 *
 * Plain pointers and sizes only.  `stream` is a cudaStream_t passed as void* (NULL = legacy
 * default stream).  Host buffers should be pinned (cudaMallocHost) for asynchronous copies.
 * The parameter set is a run-time argument `mode` in {2, 3, 5}.
 *
 * Drop-in entry points (same argument meaning, ownership and error behaviour as the reference's
 * include/api.cuh:27-63, which has one compile-time mode per library):
 *   cudil_keypair  <-> crypto_sign_keypair    (include/api.cuh:27-29, src/api.cu:26-61)
 *   cudil_sign     <-> crypto_sign_signature  (include/api.cuh:51-56, src/api.cu:63-452)
 *   cudil_verify   <-> crypto_sign_verify     (include/api.cuh:58-63, src/api.cu:454-515)
 * The per-mode C++ signatures of api.cuh are provided by include/api.cuh in this repository,
 * implemented on top of these functions.
 */
#ifndef CUDILITHIUM_B200_H
#define CUDILITHIUM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define CUDIL_OK 0
#define CUDIL_ERR_INVALID (-1)   /* bad mode, size, pitch or pointer */
#define CUDIL_ERR_CUDA (-2)      /* a CUDA call or kernel launch failed */
#define CUDIL_ERR_TIMEOUT (-3)   /* a bounded device wait gave up (fused engine) */
#define CUDIL_ERR_BUDGET (-4)    /* request exceeds the engine's device-memory budget */

typedef struct {
    int mode, k, l, eta, tau, beta, gamma1, gamma2, omega;
    int pk_bytes, sk_bytes, sig_bytes;
    int polyz_packed, polyw1_packed, polyeta_packed;
} cudil_params;

/* Layout-compatible with the reference's sign_lut_element / copy_lut_element
 * (include/api.cuh:31-39). */
typedef struct {
    int32_t done_flag;
    uint16_t nonce;
} cudil_sign_lut_element;

typedef struct {
    size_t exec_idx;
    size_t sign_idx;
} cudil_copy_lut_element;

/* The reference's task_lut (include/api.cuh:41-49) with the std::vector replaced by
 * pointer + length.  All arrays are caller-allocated: sign_lut[sign_lut_len] on the host
 * (sign_lut_len must equal batch_size), h_* pinned host arrays and d_* device arrays of
 * exec_threshold entries each. */
typedef struct {
    cudil_sign_lut_element *sign_lut;
    size_t sign_lut_len;
    uint32_t *h_exec_lut;
    uint8_t *h_done_lut;
    cudil_copy_lut_element *h_copy_lut;
    uint32_t *d_exec_lut;
    uint8_t *d_done_lut;
    cudil_copy_lut_element *d_copy_lut;
} cudil_task_lut;

/* Library / parameter queries. */
const char *cudil_version(void);
/* Text of the last CUDA failure reported as CUDIL_ERR_CUDA on the calling host thread (the CUDA
 * error string and the library source location), "no error" before any. */
const char *cudil_last_error(void);
int cudil_get_params(int mode, cudil_params *out);

/* Minimum per-item row sizes of the caller-allocated pitched pools.  They equal the reference's
 * row formulas (tests/test_vectors.cu:62-166), so pools sized for the reference fit. */
size_t cudil_keypair_row_bytes(int mode);
size_t cudil_sign_row_bytes(int mode, size_t mlen);
size_t cudil_sign_temp_row_bytes(int mode);
size_t cudil_verify_row_bytes(int mode, size_t mlen);

/* Key generation for batch_size keys; seed of key i = SHAKE128(le64(rand_index + 2i + 1))[0:32]
 * (src/keypair.cu:53-59).  pk/sk: dense host arrays.  Asynchronous on `stream`; returns after
 * queueing (results valid after the caller synchronizes), as crypto_sign_keypair. */
int cudil_keypair(int mode, uint8_t *pk, uint8_t *sk, uint8_t *d_keypair_pool, size_t keypair_pool_pitch,
                  size_t batch_size, void *stream, size_t rand_index);

/* Key generation from caller-provided 32-byte seeds (seeds: dense host array). */
int cudil_keypair_from_seed(int mode, uint8_t *pk, uint8_t *sk, const uint8_t *seeds, uint8_t *d_keypair_pool,
                            size_t keypair_pool_pitch, size_t batch_size, void *stream);

/* Deterministic signing of batch_size messages of mlen bytes; the signature of each item is the
 * one of the smallest nonce whose attempt is accepted.  Synchronizes `stream` once per rejection
 * round (as the reference, src/api.cu:307-310); the final signature copy is asynchronous. */
int cudil_sign(int mode, uint8_t *sig, size_t sig_pitch, size_t *siglen, const uint8_t *m, size_t m_pitch,
               size_t mlen, const uint8_t *sk, uint8_t *d_sign_pool, size_t sign_pool_pitch, uint8_t *d_temp_pool,
               size_t temp_pool_pitch, cudil_task_lut *lut, size_t exec_threshold, size_t batch_size, void *stream);

/* ret[i] = 0 if signature i is valid for (m_i, pk_i), else -1.  siglen != sig_bytes sets every
 * ret[i] = -1 without touching the GPU (src/api.cu:461-464).  Asynchronous on `stream`. */
int cudil_verify(int mode, int *ret, const uint8_t *sig, size_t sig_pitch, size_t siglen, const uint8_t *m,
                 size_t m_pitch, size_t mlen, const uint8_t *pk, uint8_t *d_verify_pool, size_t verify_pool_pitch,
                 size_t batch_size, void *stream);

/* Randomized signing (the reference's DILITHIUM_RANDOMIZED_SIGNING, src/api.cu:143-148): the
 * per-message seed rho' is 64 caller-supplied random bytes (row i at rhoprime + i * rhoprime_pitch)
 * instead of SHAKE256(K || mu).  The caller draws them from its random source (the api.cuh shim
 * uses the operating system's); everything else is cudil_sign / cudil_sign_dev.  Given rho', the
 * signature is deterministic (the smallest accepted nonce), so it can be checked bit for bit. */
int cudil_sign_randomized(int mode, uint8_t *sig, size_t sig_pitch, size_t *siglen, const uint8_t *m, size_t m_pitch,
                          size_t mlen, const uint8_t *sk, const uint8_t *rhoprime, size_t rhoprime_pitch,
                          uint8_t *d_sign_pool, size_t sign_pool_pitch, uint8_t *d_temp_pool, size_t temp_pool_pitch,
                          cudil_task_lut *lut, size_t exec_threshold, size_t batch_size, void *stream);
/* Device-side source of randomized-signing seeds (the reference draws rho' on the host with
 * randombytes, src/api.cu:143-148): row i of d_rhoprime (rhoprime_pitch >= 64 bytes apart, device
 * memory) = SHAKE256(seed || le64(counter + i), 64), a SHAKE256 XOF in counter mode keyed by one
 * 32-byte seed from the caller's entropy source (host memory, read during the call).  Distinct
 * (seed, counter) ranges give independent rho' values; reusing a range repeats them. */
int cudil_derive_rhoprime(uint8_t *d_rhoprime, size_t rhoprime_pitch, const uint8_t *seed, unsigned long long counter,
                          size_t n, void *stream);
int cudil_sign_dev_randomized(int mode, uint8_t *d_sig, size_t sig_pitch, const uint8_t *d_m, size_t m_pitch,
                              size_t mlen, const uint8_t *d_sk, const uint8_t *d_rhoprime, size_t rhoprime_pitch,
                              uint8_t *d_sign_pool, size_t sign_pool_pitch, uint8_t *d_temp_pool,
                              size_t temp_pool_pitch, cudil_task_lut *lut, size_t exec_threshold, size_t batch_size,
                              void *stream);

/* Signed-message format of NIST-style callers (extends the reference, which has only detached
 * signatures): sm row i = sig_i || m_i, smlen = sig_bytes + mlen.
 * cudil_crypto_sign: host buffers as cudil_sign (m may lie inside sm; rows of sm are sm_pitch
 *   apart and at least sig_bytes + mlen long).  Synchronizes `stream` once per rejection round.
 * cudil_crypto_sign_open: verifies every row of smlen bytes; ret[i] = 0 and m row i = the message
 *   if valid, else ret[i] = -1 and m row i zeroed; *mlen = smlen - sig_bytes (smlen < sig_bytes:
 *   every ret[i] = -1, *mlen = 0).  Synchronizes `stream` before releasing the messages. */
int cudil_crypto_sign(int mode, uint8_t *sm, size_t sm_pitch, size_t *smlen, const uint8_t *m, size_t m_pitch,
                      size_t mlen, const uint8_t *sk, uint8_t *d_sign_pool, size_t sign_pool_pitch,
                      uint8_t *d_temp_pool, size_t temp_pool_pitch, cudil_task_lut *lut, size_t exec_threshold,
                      size_t batch_size, void *stream);
int cudil_crypto_sign_open(int mode, uint8_t *m, size_t m_pitch, size_t *mlen, int *ret, const uint8_t *sm,
                           size_t sm_pitch, size_t smlen, const uint8_t *pk, uint8_t *d_verify_pool,
                           size_t verify_pool_pitch, size_t batch_size, void *stream);

/* Batched well-formedness checks, a parse step of their own (extends the reference, whose hint
 * checks run inside verification, src/verify.cu:51-93).  All pointers are device memory; results
 * are asynchronous on `stream`.
 * cudil_sig_check: d_status[i] bit 0 = hint encoding invalid, bit 1 = a z coefficient with
 *   |z| >= gamma1 - beta; 0 = well formed (verification still decides validity).
 * cudil_sk_check: d_status[i] = 1 if an s1 / s2 coefficient field lies outside [0, 2 eta] (dense
 *   rows of sk_bytes).  Public keys need no check: every pk_bytes string is a valid encoding. */
int cudil_sig_check(int mode, int *d_status, const uint8_t *d_sig, size_t sig_pitch, size_t batch_size, void *stream);
int cudil_sk_check(int mode, int *d_status, const uint8_t *d_sk, size_t batch_size, void *stream);

/* Device-resident variants: every data pointer is device memory (m, sk, pk, sig, seeds, ret),
 * nothing crosses PCIe except the sign scheduler's per-round flags. */
int cudil_keypair_dev(int mode, uint8_t *d_pk, uint8_t *d_sk, const uint8_t *d_seeds, uint8_t *d_keypair_pool,
                      size_t keypair_pool_pitch, size_t batch_size, void *stream, size_t rand_index);
int cudil_sign_dev(int mode, uint8_t *d_sig, size_t sig_pitch, const uint8_t *d_m, size_t m_pitch, size_t mlen,
                   const uint8_t *d_sk, uint8_t *d_sign_pool, size_t sign_pool_pitch, uint8_t *d_temp_pool,
                   size_t temp_pool_pitch, cudil_task_lut *lut, size_t exec_threshold, size_t batch_size,
                   void *stream);
int cudil_verify_dev(int mode, int *d_ret, const uint8_t *d_sig, size_t sig_pitch, size_t siglen, const uint8_t *d_m,
                     size_t m_pitch, size_t mlen, const uint8_t *d_pk, uint8_t *d_verify_pool,
                     size_t verify_pool_pitch, size_t batch_size, void *stream);

/* Per-item message lengths (device-resident variants; extends the reference API, which has one
 * mlen per call, include/api.cuh:51-63): row i of d_m (m_pitch apart) holds a message of
 * d_mlens[i] <= max_mlen bytes; pools are sized for max_mlen. */
int cudil_sign_dev_varlen(int mode, uint8_t *d_sig, size_t sig_pitch, const uint8_t *d_m, size_t m_pitch,
                          const uint32_t *d_mlens, size_t max_mlen, const uint8_t *d_sk, uint8_t *d_sign_pool,
                          size_t sign_pool_pitch, uint8_t *d_temp_pool, size_t temp_pool_pitch, cudil_task_lut *lut,
                          size_t exec_threshold, size_t batch_size, void *stream);
int cudil_verify_dev_varlen(int mode, int *d_ret, const uint8_t *d_sig, size_t sig_pitch, size_t siglen,
                            const uint8_t *d_m, size_t m_pitch, const uint32_t *d_mlens, size_t max_mlen,
                            const uint8_t *d_pk, uint8_t *d_verify_pool, size_t verify_pool_pitch, size_t batch_size,
                            void *stream);

/* Verification without any device allocation, for callers that may not allocate device memory
 * where they verify (budgeted or pre-reserved device memory, latency-critical threads that must
 * not hit cudaMalloc/cudaFree, hosts that own every allocation).  No counterpart in the
 * reference (its crypto_sign_verify needs a caller-allocated pool).  Same arguments and results as
 * cudil_verify minus the pool: the pool is a fixed CUDIL_NOALLOC_SCRATCH_BYTES array inside the
 * library, reserved on every GPU that loads it.  At most cudil_verify_noalloc_max_batch(mode,
 * mlen) signatures per call (larger batches: CUDIL_ERR_BUDGET).  All calls share the array, so
 * calls that overlap on the GPU race and must be serialized by the caller.  The first call on a
 * device looks up the array's address; make it before any stream capture. */
#define CUDIL_NOALLOC_SCRATCH_BYTES ((size_t)16 << 20)
size_t cudil_verify_noalloc_max_batch(int mode, size_t mlen);
int cudil_verify_noalloc(int mode, int *ret, const uint8_t *sig, size_t sig_pitch, size_t siglen, const uint8_t *m,
                         size_t m_pitch, size_t mlen, const uint8_t *pk, size_t batch_size, void *stream);

/* NTT microbenchmark (no reference API counterpart; replaces benches/bench_ntt_radix{2,8}.cu):
 * d_out[p] = invNTT(NTT(d_a[p]) o d_b[p]) for npolys polynomials of 256 int32, Montgomery
 * pointwise product, bit-exact with the oracle's ntt / poly_pointwise_montgomery /
 * invntt_tomont.  d_out may alias d_a. */
int cudil_ntt_mul(const int32_t *d_a, const int32_t *d_b, int32_t *d_out, size_t npolys, void *stream);

/* ---------------------------------------------------------------------------------------------
 * Fused engine (no reference counterpart; the reference re-expands A and re-transforms the
 * secret key for every sign call and drives every rejection round from the host).
 *
 * One engine serves one parameter set on the current device.  It keeps, per key, the expanded
 * matrix A_hat and the NTT-domain key material resident in device memory (secret keys: A_hat,
 * s1_hat, s2_hat, t0_hat, rho, K, tr; public keys: A_hat, NTT(t1 * 2^d), tr) and runs a whole
 * signing batch as one CUDA-graph launch around ONE persistent kernel whose device-side ticket
 * queue hands every rejected attempt's slot the next (message, nonce) attempt.  Results are
 * identical to cudil_sign / cudil_verify (deterministic signing: smallest accepted nonce).
 *
 * create:  allocates everything up front (max_keys cache rows of each kind, max_items messages per
 *          batch, scratch for one persistent grid); CUDIL_ERR_BUDGET if that exceeds
 *          device_budget_bytes (0 = no limit).  threads_per_block: 128 or 256 (0 = 256).
 * sign/verify: d_msgs is one device buffer of msgs_bytes bytes holding every message at an 8-byte
 *          aligned offset (offsets[i] + mlens[i] <= msgs_bytes, checked before any launch);
 *          offsets / mlens / key_idx are HOST arrays of n entries (uploaded before the launch);
 *          signatures are dense (sig_bytes each).  The signature output of sign may be device
 *          memory or pinned host memory: in host memory each signature is written over PCIe as
 *          soon as it is found, so the download overlaps the signing (pageable host memory:
 *          CUDIL_ERR_INVALID).  Asynchronous on `stream`; one batch in flight
 *          per engine (calls on one engine must be ordered on one stream).
 * last_status: attempts and error flags of the last completed batch (valid after sync);
 *          returns CUDIL_ERR_TIMEOUT if a device-side loop hit its bound (cudil_engine_set_limits).
 *          Error bits: 1 = a per-item publication-lock wait gave up (that attempt's signature is
 *          not written); 2 = an item reached its nonce limit (if none of its nonces was accepted,
 *          its row is not written and cudil_engine_last_nonces reports CUDIL_NONCE_EXHAUSTED); 4 = an
 *          asynchronous signer block gave up after its idle-poll limit (its pending items stay
 *          unsigned).  The engine stays usable after any of them. */
typedef struct cudil_engine cudil_engine;
int cudil_engine_create(cudil_engine **out, int mode, size_t max_keys, size_t max_items, int threads_per_block,
                        size_t device_budget_bytes);
int cudil_engine_destroy(cudil_engine *e);
size_t cudil_engine_device_bytes(const cudil_engine *e);
int cudil_engine_set_secret_keys(cudil_engine *e, const uint8_t *d_sk, size_t nkeys, void *stream);
/* Builds the cache rows of keys first .. first + nkeys - 1 from nkeys packed secret keys at d_sk
 * (first must not exceed the number of rows built so far, so the built rows stay a prefix), e.g.
 * to replace some keys of a resident table, or to build the table in chunks, each chunk's build
 * queued behind its own host-to-device copy so the copies of later chunks overlap it. */
int cudil_engine_update_secret_keys(cudil_engine *e, const uint8_t *d_sk, size_t first, size_t nkeys, void *stream);
/* Share src's key caches (same parameter set; src must outlive e).  An engine created with
 * max_keys = 0 owns no caches and must attach before signing or verifying.  Each sign or verify
 * call of e uses the key rows the owning engine has built by then, so keys may be set on the owner
 * before or after attaching (in stream order with e's work, as for the owner's own calls). */
int cudil_engine_attach_keys(cudil_engine *e, const cudil_engine *src);
int cudil_engine_set_public_keys(cudil_engine *e, const uint8_t *d_pk, size_t nkeys, void *stream);
int cudil_engine_sign(cudil_engine *e, uint8_t *d_sig, const uint8_t *d_msgs, size_t msgs_bytes,
                      const unsigned long long *offsets, const uint32_t *mlens, const uint32_t *key_idx, size_t n,
                      void *stream);
/* Randomized signing through the engine: d_rhoprime holds 64 random bytes per item (dense, device
 * memory), used as rho' instead of SHAKE256(K || mu). */
int cudil_engine_sign_randomized(cudil_engine *e, uint8_t *d_sig, const uint8_t *d_msgs, size_t msgs_bytes,
                                 const unsigned long long *offsets, const uint32_t *mlens, const uint32_t *key_idx,
                                 const uint8_t *d_rhoprime, size_t n, void *stream);
/* Seeded randomized signing through the engine: rho' of item i is derived on the device as
 * SHAKE256(rho_seed || le64(rho_counter + i), 64) (cudil_derive_rhoprime's rule) inside the
 * batch's prehash kernel; rho_seed is 32 bytes of host memory read during the call. */
int cudil_engine_sign_seeded(cudil_engine *e, uint8_t *d_sig, const uint8_t *d_msgs, size_t msgs_bytes,
                             const unsigned long long *offsets, const uint32_t *mlens, const uint32_t *key_idx,
                             const uint8_t *rho_seed, unsigned long long rho_counter, size_t n, void *stream);
int cudil_engine_verify(cudil_engine *e, int *d_ret, const uint8_t *d_sig, const uint8_t *d_msgs, size_t msgs_bytes,
                        const unsigned long long *offsets, const uint32_t *mlens, const uint32_t *key_idx, size_t n,
                        void *stream);
int cudil_engine_last_status(const cudil_engine *e, unsigned long long *attempts, unsigned *error);
/* Bounds of the signer's device-side loops, from the next signing batch on (the defaults below):
 *   nonce_limit  nonces an item may try (1 .. 65536; the reference's 16-bit nonce field allows
 *                65536, src/api.cu:224 packs it into the low 16 bits of an exec slot);
 *   lock_spins   tries for an item's publication lock before the attempt gives up (0 = at once);
 *   idle_polls   empty polls before an asynchronous signer block gives up (0 = at the first).
 * Running into a bound sets an error bit of cudil_engine_last_status instead of waiting longer. */
#define CUDIL_ENGINE_NONCE_LIMIT 65536u
#define CUDIL_ENGINE_LOCK_SPINS (1u << 22)
#define CUDIL_ENGINE_IDLE_POLLS (1u << 21)
int cudil_engine_set_limits(cudil_engine *e, unsigned nonce_limit, unsigned lock_spins, unsigned idle_polls);
/* Winning (smallest accepted) nonce of each of the first n items of the last signing batch, copied
 * into out (host or device memory) on `stream`; returns once the copy has completed.  Deterministic
 * signing ran nonce + 1 attempts for the item; CUDIL_NONCE_EXHAUSTED marks an item whose nonces ran
 * out (error bit 2). */
#define CUDIL_NONCE_EXHAUSTED 0xFFFFFFFEu
int cudil_engine_last_nonces(cudil_engine *e, unsigned *out, size_t n, void *stream);
/* Work counters of the last completed signing batch: attempts run and inverse NTTs executed by the
 * rejection checks (for throughput accounting). */
int cudil_engine_last_work(const cudil_engine *e, unsigned long long *attempts, unsigned long long *reject_intt);
/* Signer tuning: per-block target of signing attempts in flight (1 .. 2 * threads_per_block).
 * Every block owns a share of the batch's items; while it has many pending items each has at most
 * two attempts in flight, and as they run out the remaining ones get up to target / pending
 * consecutive nonces in flight (at most 64).  0 = default (threads_per_block).  Takes effect
 * from the next batch. */
int cudil_engine_set_spec_slots(cudil_engine *e, unsigned spec_slots);
/* Signer kernel: 0 (default) = phased persistent kernel (block-wide Keccak / NTT phases,
 * threads_per_block threads); 1..4 = asynchronous persistent kernel -- warps take ready jobs from a
 * per-block attempt-slot state machine without block barriers, the speculation target capped at
 * the slot count -- with (threads, slots) per block of (256, 64), (512, 128), (640, 160) and
 * (768, 192); 5 = the phased kernel with one wide block per SM (512 threads; 384 for Dilithium5).
 * Results are identical for every variant. */
int cudil_engine_set_sign_kernel(cudil_engine *e, int variant);
/* Large batches: a signing batch of at least min_items items runs signer kernel `variant` with
 * speculation target `spec_slots` (0 = threads_per_block) through a graph of its own; smaller
 * batches keep the kernel and target set above.  min_items = 0 turns the large-batch choice off.
 * Default: min_items = 224 items per SM, variant 5 (the wide phased kernel), target 128, which is
 * the fastest signer at 64 Ki items for every parameter set.  Results are identical either way. */
int cudil_engine_set_large_batch(cudil_engine *e, size_t min_items, int variant, unsigned spec_slots);
/* Job profile of the last batch of the asynchronous signer, summed over warps: SM cycles spent in
 * rejection / w / challenge / ExpandMask jobs, claims and idle polls (out[0..5]) and their counts
 * (out[6..11]; challenge and ExpandMask count attempts). */
int cudil_engine_last_jobs(const cudil_engine *e, unsigned long long out[12]);
/* Signer phase profile of the last batch: SM cycles summed over blocks spent in slot refills,
 * Keccak phases, NTT phases and in total, and the number of block iterations. */
int cudil_engine_last_phases(const cudil_engine *e, unsigned long long cycles[4], unsigned *iterations);
int cudil_engine_info(const cudil_engine *e, int *mode, int *threads, int *sign_blocks, int *verify_blocks);

/* ---------------------------------------------------------------------------------------------
 * Request server: continuous batching over a mixed request stream (no reference counterpart; the
 * reference only has the blocking batch calls above).
 *
 * cudil_serve_trace replays an open-loop trace in real time on the current device.  Request i
 * becomes visible arrival_s seconds after the start and queues in the FIFO of its (parameter set,
 * operation) lane.  Each lane owns up to slots_per_lane batch slots (stream + device buffers, more
 * for busy lanes with lane_slots_by_load); a
 * free slot takes everything queued in its lane (at most max_batch) as one batch, so batches of
 * every lane overlap on the device while new requests queue.  Slots are created only while the
 * device-memory estimate stays within device_budget_bytes (0 = unlimited); every lane in use
 * needs one (else CUDIL_ERR_BUDGET).
 * path 0: fused engines sharing one resident key cache per parameter set (sk and pk of every key
 *         expanded once before the replay starts, outside the timed region);
 * path 1: the plain stage-by-stage calls (key material expanded per batch).
 * Messages are msgs[msg_off .. msg_off + mlen) (mlen <= max_mlen); verify requests read
 * sigs[sig_off .. + sig_bytes).  Results: status 0 / -1 (verify), done_s = host time the request's
 * batch completed; signatures go to sig_out + i * sig_out_pitch (NULL: not returned).
 * Returns CUDIL_OK or the first error. */
typedef struct {
    double arrival_s;
    int32_t mode; /* 2, 3 or 5 */
    int32_t op;   /* 0 sign, 1 verify */
    uint32_t key; /* index into the parameter set's key array */
    uint32_t mlen;
    unsigned long long msg_off, sig_off;
} cudil_request;

typedef struct {
    double done_s;
    int32_t status;
    uint32_t batch_size; /* size of the batch that served the request */
} cudil_request_result;

typedef struct {
    size_t device_budget_bytes;
    int32_t path;           /* 0 fused, 1 plain */
    int32_t slots_per_lane; /* >= 1 */
    int32_t max_batch;      /* >= 1 */
    int32_t engine_threads; /* fused: threads per block (0 = default) */
    int32_t engine_spec_slots;    /* fused: signer speculation target (0 = default) */
    int32_t plain_exec_threshold; /* plain: signing attempts per round (>= 1) */
    uint32_t max_mlen;
    /* 0: every lane gets slots_per_lane slots; 1: a lane gets slots in proportion to its share of
     * the trace's requests, round(share * slots_per_lane * lanes), at least slots_per_lane (a lane
     * that carries most of the requests also needs more host threads staging its batches) */
    uint32_t lane_slots_by_load;
} cudil_serve_config;

typedef struct {
    double wall_s;       /* first arrival window start to last completion */
    size_t batches;      /* batches launched */
    size_t slots;        /* batch slots created within the budget */
    size_t device_bytes; /* device-memory estimate of caches + slots */
    /* summed over slots: staging requests into pinned buffers, first copy / launch to stream
     * completion (H2D + kernels + D2H, including waits behind other slots), result write-back */
    double host_stage_s, device_wait_s, host_post_s;
} cudil_serve_stats;

int cudil_serve_trace(const cudil_serve_config *cfg, const uint8_t *const sk[3], const uint8_t *const pk[3],
                      const size_t nkeys[3], const cudil_request *reqs, size_t nreq, const uint8_t *msgs,
                      const uint8_t *sigs, uint8_t *sig_out, size_t sig_out_pitch, cudil_request_result *results,
                      cudil_serve_stats *stats);

/* Peak of the 32-bit LOP3/funnel-shift mix Keccak-f[1600] issues: launches `blocks` x 256 threads
 * doing `iters` x 32 ALU operations each; *ops_per_launch receives the operation count. */
int cudil_alu_peak(uint32_t *d_out, int blocks, int iters, void *stream, double *ops_per_launch);

/* Bounds-checked build (libcudilithium_b200_bc.so, built with `python cudilithium_b200/build.py
 * --bounds-check`): device-side range checks of pool rows, attempt slots, item indices and key-cache
 * rows record the first failing check's site code and skip the access instead of trapping.
 * cudil_bounds_check_status stores that code in *error (0 = every check passed since the last
 * reset) and clears it when reset != 0; in the normal library it returns CUDIL_ERR_INVALID. */
int cudil_bounds_check_status(unsigned *error, int reset);

/* Launch accounting.  cudil_launch_count: kernels launched by this library so far (process-wide).
 * cudil_kernel_timing(1) brackets every later launch with CUDA events on its stream (off by
 * default); cudil_kernel_stats returns the accumulated device time and launches of kernel id
 * (0 <= id < cudil_kernel_count(), named by cudil_kernel_name). */
unsigned long long cudil_launch_count(void);
void cudil_kernel_timing(int enable);
int cudil_kernel_count(void);
const char *cudil_kernel_name(int id);
int cudil_kernel_stats(int id, double *total_ms, unsigned long long *launches);
void cudil_kernel_stats_reset(void);

#ifdef __cplusplus
}
#endif
#endif
