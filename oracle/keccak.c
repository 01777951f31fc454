/*
 * CPU oracle (test infrastructure only; never linked into the product path).
 *
 * Keccak-f[1600] and the SHAKE128 / SHAKE256 extendable-output functions, restated
 * from FIPS 202 (sections 3.2 and 6.2).  The reference's own CPU copy lives in
 * src/fips202/fips202.c (KeccakF1600_StatePermute :83, keccak_absorb_once :457,
 * keccak_squeezeblocks :495, shake128 :682, shake256 :704); this file follows the same
 * byte conventions (little-endian lanes, pad byte 0x1F, final bit 0x80 of the rate)
 * but derives the round constants and rotation offsets from the specification's
 * LFSR and (t+1)(t+2)/2 rules at first use instead of carrying tables.
 *
 * Parity: the oracle built on this file reproduces the reference's pinned test-vector
 * digests (tests/CMakeLists.txt:21-23 of the reference); the Keccak itself is also
 * cross-checked byte-for-byte against the reference's fips202.c when that file is
 * compiled into oracle/_ref/.
 */
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#include "oracle.h"

static uint64_t g_rc[24];
static unsigned g_rot[25];
static unsigned g_pi_src[25]; /* B[dst] = rot(A[g_pi_src[dst]]) */
static int g_ready = 0;

/* rc(t) from FIPS 202 Algorithm 5: LFSR x^8 + x^6 + x^5 + x^4 + 1. */
static int rc_bit(unsigned t) {
    unsigned r = 1, i;
    if (t % 255 == 0) return 1;
    for (i = 1; i <= t % 255; i++) {
        r <<= 1;
        if (r & 0x100) r ^= 0x171;
    }
    return r & 1;
}

/* Runs once when the library is loaded, before any caller can start threads: a lazy first-use
 * initialisation raced when the first permutations ran on several OpenMP threads at once (a second
 * initialiser cleared g_rot while a first thread was already permuting with it). */
__attribute__((constructor)) static void keccak_tables_init(void) {
    unsigned ir, j, t, x, y;
    if (g_ready) return;
    for (ir = 0; ir < 24; ir++) {
        uint64_t rc = 0;
        for (j = 0; j <= 6; j++)
            if (rc_bit(j + 7 * ir)) rc |= 1ULL << ((1u << j) - 1);
        g_rc[ir] = rc;
    }
    /* rho offsets: walk (x,y) <- (y, 2x+3y) from (1,0), offset (t+1)(t+2)/2 mod 64. */
    memset(g_rot, 0, sizeof g_rot);
    x = 1;
    y = 0;
    for (t = 0; t < 24; t++) {
        unsigned nx = y, ny = (2 * x + 3 * y) % 5;
        g_rot[x + 5 * y] = ((t + 1) * (t + 2) / 2) % 64;
        x = nx;
        y = ny;
    }
    /* pi: A'[x,y] = A[(x+3y) mod 5, x]. */
    for (y = 0; y < 5; y++)
        for (x = 0; x < 5; x++) g_pi_src[x + 5 * y] = ((x + 3 * y) % 5) + 5 * x;
    g_ready = 1;
}

static inline uint64_t rol64(uint64_t v, unsigned n) { return n ? (v << n) | (v >> (64 - n)) : v; }

void ora_keccak_f1600(uint64_t s[25]) {
    uint64_t c[5], d[5], b[25];
    unsigned r, x, y, i;
    if (!g_ready) keccak_tables_init();
    for (r = 0; r < 24; r++) {
        for (x = 0; x < 5; x++) c[x] = s[x] ^ s[x + 5] ^ s[x + 10] ^ s[x + 15] ^ s[x + 20];
        for (x = 0; x < 5; x++) d[x] = c[(x + 4) % 5] ^ rol64(c[(x + 1) % 5], 1);
        for (i = 0; i < 25; i++) s[i] ^= d[i % 5];
        for (i = 0; i < 25; i++) b[i] = rol64(s[g_pi_src[i]], g_rot[g_pi_src[i]]);
        for (y = 0; y < 5; y++)
            for (x = 0; x < 5; x++)
                s[x + 5 * y] = b[x + 5 * y] ^ (~b[(x + 1) % 5 + 5 * y] & b[(x + 2) % 5 + 5 * y]);
        s[0] ^= g_rc[r];
    }
}

void ora_xof_init(ora_xof *st, unsigned rate) {
    memset(st->s, 0, sizeof st->s);
    st->pos = 0;
    st->rate = rate;
    st->squeezing = 0;
    if (!g_ready) keccak_tables_init();
}

void ora_xof_absorb(ora_xof *st, const uint8_t *in, size_t inlen) {
    size_t i;
    for (i = 0; i < inlen; i++) {
        st->s[st->pos / 8] ^= (uint64_t)in[i] << (8 * (st->pos % 8));
        if (++st->pos == st->rate) {
            ora_keccak_f1600(st->s);
            st->pos = 0;
        }
    }
}

void ora_xof_finalize(ora_xof *st) {
    st->s[st->pos / 8] ^= (uint64_t)0x1F << (8 * (st->pos % 8));
    st->s[(st->rate - 1) / 8] ^= 1ULL << 63;
    st->pos = st->rate; /* forces a permutation before the first output byte */
    st->squeezing = 1;
}

void ora_xof_squeeze(ora_xof *st, uint8_t *out, size_t outlen) {
    size_t i;
    for (i = 0; i < outlen; i++) {
        if (st->pos == st->rate) {
            ora_keccak_f1600(st->s);
            st->pos = 0;
        }
        out[i] = (uint8_t)(st->s[st->pos / 8] >> (8 * (st->pos % 8)));
        st->pos++;
    }
}

void ora_shake128(uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen) {
    ora_xof st;
    ora_xof_init(&st, ORA_SHAKE128_RATE);
    ora_xof_absorb(&st, in, inlen);
    ora_xof_finalize(&st);
    ora_xof_squeeze(&st, out, outlen);
}

void ora_shake256(uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen) {
    ora_xof st;
    ora_xof_init(&st, ORA_SHAKE256_RATE);
    ora_xof_absorb(&st, in, inlen);
    ora_xof_finalize(&st);
    ora_xof_squeeze(&st, out, outlen);
}
