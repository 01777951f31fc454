/*
 * CPU oracle for the batched Dilithium (round 3, v3.1) hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the cpu_baseline /
 * --impl reference legs of bench.py may load this library, and only as the checker or the
 * timed CPU baseline.  The product (cudilithium_b200) never links or calls it.
 *
 * The parameter set is a runtime argument (2, 3 or 5) instead of the reference's
 * compile-time DILITHIUM_MODE (include/params.h:14-45 of the reference).
 */
#ifndef CUDIL_ORACLE_H
#define CUDIL_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORA_SHAKE128_RATE 168
#define ORA_SHAKE256_RATE 136
#define ORA_N 256
#define ORA_Q 8380417
#define ORA_SEEDBYTES 32
#define ORA_CRHBYTES 64

typedef struct {
    uint64_t s[25];
    unsigned pos;
    unsigned rate;
    int squeezing;
} ora_xof;

typedef struct {
    int mode;
    int k, l, eta, tau, beta, gamma1, gamma2, omega;
    int polyz_packed, polyw1_packed, polyeta_packed;
    int pk_bytes, sk_bytes, sig_bytes;
} ora_params;

/* keccak.c */
void ora_keccak_f1600(uint64_t s[25]);
void ora_xof_init(ora_xof *st, unsigned rate);
void ora_xof_absorb(ora_xof *st, const uint8_t *in, size_t inlen);
void ora_xof_finalize(ora_xof *st);
void ora_xof_squeeze(ora_xof *st, uint8_t *out, size_t outlen);
void ora_shake128(uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen);
void ora_shake256(uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen);

/* dilithium.c */
int ora_params_get(int mode, ora_params *p);

/* Single operations. */
int ora_keypair_from_seed(int mode, uint8_t *pk, uint8_t *sk, const uint8_t seed[32]);
int ora_sign(int mode, uint8_t *sig, const uint8_t *m, size_t mlen, const uint8_t *sk, int *attempts);
int ora_sign_rhoprime(int mode, uint8_t *sig, const uint8_t *m, size_t mlen, const uint8_t *sk,
                      const uint8_t *rhoprime, int *attempts);
int ora_verify(int mode, const uint8_t *sig, size_t siglen, const uint8_t *m, size_t mlen, const uint8_t *pk);
int ora_sig_check(int mode, const uint8_t *sig);
int ora_hint_check(int mode, const uint8_t *sig, int xor_lanes);
void ora_derive_rhoprime(uint8_t *out, const uint8_t seed[32], uint64_t counter, size_t n);
int ora_verify_xor_ballots(int mode, const uint8_t *sig, size_t siglen, const uint8_t *m, size_t mlen,
                           const uint8_t *pk);
int ora_sk_check(int mode, const uint8_t *sk);

/* Batched forms (OpenMP over items; nthreads <= 0 means all available). */
void ora_seed_from_ctr(uint8_t seed[32], uint64_t ctr);
int ora_keypair_batch(int mode, uint8_t *pk, uint8_t *sk, size_t n, uint64_t rand_index, int nthreads);
int ora_keypair_seeds_batch(int mode, uint8_t *pk, uint8_t *sk, const uint8_t *seeds, size_t n, int nthreads);
int ora_sign_batch(int mode, uint8_t *sig, size_t sig_pitch, const uint8_t *m, size_t m_pitch,
                   const uint64_t *mlens, const uint8_t *sk, size_t sk_pitch, size_t n, int nthreads,
                   int32_t *attempts);
int ora_verify_batch(int mode, int32_t *ret, const uint8_t *sig, size_t sig_pitch, size_t siglen,
                     const uint8_t *m, size_t m_pitch, const uint64_t *mlens, const uint8_t *pk, size_t pk_pitch,
                     size_t n, int nthreads);

/* Stage-level entry points used by the parity tests. */
void ora_ntt(int32_t a[256]);
void ora_invntt_tomont(int32_t a[256]);
int32_t ora_montgomery_reduce(int64_t a);
void ora_ntt_mul_batch(int32_t *a, const int32_t *b, size_t n, int nthreads);
void ora_expand_a(int mode, int32_t *mat, const uint8_t rho[32]);
void ora_expand_mask(int mode, int32_t *y, const uint8_t rhoprime[64], uint16_t nonce);
void ora_challenge(int mode, int32_t c[256], const uint8_t seed[32]);

/* Test-vector file in the reference's tests/test_vectors.cu format (10000 items, MLEN=32). */
long ora_tvecs(int mode, size_t nvectors, char *buf, size_t buflen, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
