// extern "C" boundary: run-time parameter-set dispatch onto the per-mode instantiations, pool row
// size queries, and the NTT microbenchmark kernel.
#include <climits>
#include <cstdio>
#include <cstring>
#include <cuda_runtime.h>

#include "../../include/cudilithium.h"
#include "host_impl.cuh"
#include "parse_kernels.cuh"
#include "profiling.cuh"

namespace cudil {
extern template struct Impl<2>;
extern template struct Impl<3>;
extern template struct Impl<5>;
cudaError_t bounds_status_mode2(unsigned *out, bool reset);
cudaError_t bounds_status_mode3(unsigned *out, bool reset);
cudaError_t bounds_status_mode5(unsigned *out, bool reset);

// Peak of the 32-bit logic/shift mix that Keccak-f[1600] issues (3 LOP3 : 1 funnel shift, the
// ratio of a LOP3/SHF lowering of theta/rho/chi): 8 independent chains per thread.
__global__ void __launch_bounds__(256) k_alu_peak(uint32_t *out, int iters) {
    uint32_t a[8];
    const uint32_t b = threadIdx.x * 0x9E3779B9u + 1u, c = blockIdx.x * 0x7F4A7C15u + 3u;
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = threadIdx.x + (uint32_t)k * 0x01234567u;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            uint32_t x = a[k];
            asm("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(x) : "r"(b), "r"(c));
            asm("lop3.b32 %0, %0, %1, %2, 0xD2;" : "+r"(x) : "r"(c), "r"(b));
            asm("lop3.b32 %0, %0, %1, %2, 0x78;" : "+r"(x) : "r"(b), "r"(c));
            asm("shf.l.wrap.b32 %0, %0, %1, 7;" : "+r"(x) : "r"(b));
            a[k] = x;
        }
    }
    uint32_t r = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) r ^= a[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = r;
}

// Seeded randomized signing: row i of out (pitch bytes apart) = SHAKE256(seed || le64(counter + i),
// 64), one thread per row; the seed travels by value in the kernel arguments.
struct Seed32 {
    uint32_t w[8];
};

__global__ void __launch_bounds__(kBlock) k_derive_rhoprime(uint8_t *out, size_t pitch, Seed32 seed,
                                                            unsigned long long counter, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint2 rp[8];
    derive_rhoprime(rp, seed.w, counter + (unsigned long long)i);
    uint8_t *row = out + (size_t)i * pitch;
    if ((reinterpret_cast<uintptr_t>(row) & 7u) == 0u) {
#pragma unroll
        for (int w = 0; w < 8; ++w) reinterpret_cast<uint2 *>(row)[w] = rp[w];
    } else {
#pragma unroll
        for (int w = 0; w < 8; ++w)
#pragma unroll
            for (int b = 0; b < 8; ++b) row[8 * w + b] = (uint8_t)((b < 4 ? rp[w].x >> (8 * b) : rp[w].y >> (8 * (b - 4))));
    }
}

// out = invNTT(NTT(a) o b) for npolys polynomial pairs.  A grid of a few blocks per SM walks the
// batch: each 16-thread group takes every total_groups-th polynomial, and while it transforms one it
// already has the loads of the next a (issued before the inverse transform) and of the current b
// (issued before the forward transform) in flight, so HBM latency overlaps the arithmetic.  The
// group positions' register-local twiddles come from a shared-memory copy of the table, read with
// eight 128-bit loads per transform: holding both directions' rows in registers across the loop
// would take 64 registers.
__global__ void __launch_bounds__(kBlock) k_ntt_mul(const int32_t *a, const int32_t *b, int32_t *out, long long npolys) {
    __shared__ int32_t sm[kGroupsPerBlock * NTT_SMEM_WORDS];
    // twiddle rows (forward, inverse) of the 16 group positions; chunk c (16 bytes) of row t is
    // stored at chunk (c + t) mod 8, so that the positions' reads of one chunk spread over the banks
    __shared__ __align__(16) int4 s_tw[2][16][8];
    for (int k = threadIdx.x; k < 2 * 16 * 8; k += blockDim.x) {
        const int dir = k >> 7, t = (k >> 3) & 15, c = k & 7;
        const int4 *src = reinterpret_cast<const int4 *>(dir ? g_group_tw.inv[t] : g_group_tw.fwd[t]);
        s_tw[dir][t][(c + t) & 7] = src[c];
    }
    __syncthreads();
    const long long groups = (long long)gridDim.x * (blockDim.x >> 4);
    long long p = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    if (p >= npolys) return;
    Group g = make_group(sm, threadIdx.x >> 4);
    auto tw_row = [&](int dir, int2 (&tw)[16]) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int4 v = s_tw[dir][g.t][(c + g.t) & 7];
            tw[2 * c] = make_int2(v.x, v.y);
            tw[2 * c + 1] = make_int2(v.z, v.w);
        }
    };
    int32_t x[16], y[16];
    load16_strided(x, a + p * N, g.t);
#pragma unroll 1
    for (; p < npolys; p += groups) {
        load16_contig(y, b + p * N + 16 * g.t);
        {
            int2 tw[16];
            tw_row(0, tw);
            ntt16_tw<false>(x, g.sm, g.gmask, g.t, tw);
        }
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = montmul(x[m], y[m]);
        const long long nx = p + groups;
        int32_t xn[16];
        if (nx < npolys) load16_strided(xn, a + nx * N, g.t);
        {
            int2 tw[16];
            tw_row(1, tw);
            intt16_tw<false>(x, g.sm, g.gmask, g.t, tw);
        }
        store16_strided(out + p * N, x, g.t);
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = xn[m];
    }
}
}  // namespace cudil

using namespace cudil;

#define CUDIL_DISPATCH(mode, call)          \
    switch (mode) {                         \
        case 2: {                           \
            using I = Impl<2>;              \
            return call;                    \
        }                                   \
        case 3: {                           \
            using I = Impl<3>;              \
            return call;                    \
        }                                   \
        case 5: {                           \
            using I = Impl<5>;              \
            return call;                    \
        }                                   \
        default:                            \
            return CUDIL_ERR_INVALID;       \
    }

#define CUDIL_SIZE_DISPATCH(mode, expr)     \
    switch (mode) {                         \
        case 2: {                           \
            using LY = Layout<2>;           \
            return expr;                    \
        }                                   \
        case 3: {                           \
            using LY = Layout<3>;           \
            return expr;                    \
        }                                   \
        case 5: {                           \
            using LY = Layout<5>;           \
            return expr;                    \
        }                                   \
        default:                            \
            return 0;                       \
    }

template <int MODE>
static void fill_params(cudil_params *o) {
    using PM = P<MODE>;
    o->mode = MODE;
    o->k = PM::K;
    o->l = PM::L;
    o->eta = PM::ETA;
    o->tau = PM::TAU;
    o->beta = PM::BETA;
    o->gamma1 = PM::GAMMA1;
    o->gamma2 = PM::GAMMA2;
    o->omega = PM::OMEGA;
    o->pk_bytes = PM::PK_BYTES;
    o->sk_bytes = PM::SK_BYTES;
    o->sig_bytes = PM::SIG_BYTES;
    o->polyz_packed = PM::POLYZ_PACKED;
    o->polyw1_packed = PM::POLYW1_PACKED;
    o->polyeta_packed = PM::POLYETA_PACKED;
}

namespace cudil {
static thread_local char g_last_error[256] = "no error";

int cudil_record_cuda_error(cudaError_t e, const char *file, int line) {
    const char *base = file;
    for (const char *p = file; *p; ++p)
        if (*p == '/') base = p + 1;
    std::snprintf(g_last_error, sizeof g_last_error, "%s (%s:%d)", cudaGetErrorString(e), base, line);
    return CUDIL_ERR_CUDA;
}
}  // namespace cudil

extern "C" {

const char *cudil_version(void) { return "cudilithium_b200 0.1 (Dilithium round 3 v3.1, sm_100a)"; }

const char *cudil_last_error(void) { return cudil::g_last_error; }

int cudil_get_params(int mode, cudil_params *out) {
    if (!out) return CUDIL_ERR_INVALID;
    switch (mode) {
        case 2: fill_params<2>(out); return CUDIL_OK;
        case 3: fill_params<3>(out); return CUDIL_OK;
        case 5: fill_params<5>(out); return CUDIL_OK;
        default: return CUDIL_ERR_INVALID;
    }
}

size_t cudil_keypair_row_bytes(int mode) { CUDIL_SIZE_DISPATCH(mode, LY::ref_keypair_row()) }
size_t cudil_sign_row_bytes(int mode, size_t mlen) { CUDIL_SIZE_DISPATCH(mode, LY::ref_sign_row(mlen)) }
size_t cudil_sign_temp_row_bytes(int mode) { CUDIL_SIZE_DISPATCH(mode, LY::ref_sign_temp_row()) }
size_t cudil_verify_row_bytes(int mode, size_t mlen) { CUDIL_SIZE_DISPATCH(mode, LY::ref_verify_row(mlen)) }

int cudil_keypair(int mode, uint8_t *pk, uint8_t *sk, uint8_t *d_pool, size_t pitch, size_t batch, void *stream,
                  size_t rand_index) {
    CUDIL_DISPATCH(mode, I::keypair(pk, sk, nullptr, d_pool, pitch, batch, (cudaStream_t)stream, rand_index,
                                    cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost))
}

int cudil_keypair_from_seed(int mode, uint8_t *pk, uint8_t *sk, const uint8_t *seeds, uint8_t *d_pool, size_t pitch,
                            size_t batch, void *stream) {
    if (!seeds) return CUDIL_ERR_INVALID;
    CUDIL_DISPATCH(mode, I::keypair(pk, sk, seeds, d_pool, pitch, batch, (cudaStream_t)stream, 0, cudaMemcpyHostToDevice,
                                    cudaMemcpyDeviceToHost))
}

int cudil_keypair_dev(int mode, uint8_t *d_pk, uint8_t *d_sk, const uint8_t *d_seeds, uint8_t *d_pool, size_t pitch,
                      size_t batch, void *stream, size_t rand_index) {
    CUDIL_DISPATCH(mode, I::keypair(d_pk, d_sk, d_seeds, d_pool, pitch, batch, (cudaStream_t)stream, rand_index,
                                    cudaMemcpyDeviceToDevice, cudaMemcpyDeviceToDevice))
}

int cudil_sign(int mode, uint8_t *sig, size_t sig_pitch, size_t *siglen, const uint8_t *m, size_t m_pitch, size_t mlen,
               const uint8_t *sk, uint8_t *d_sign_pool, size_t sign_pitch, uint8_t *d_temp_pool, size_t temp_pitch,
               cudil_task_lut *lut, size_t exec_threshold, size_t batch, void *stream) {
    CUDIL_DISPATCH(mode, I::sign(sig, sig_pitch, siglen, m, m_pitch, mlen, sk, I::PM::SK_BYTES, d_sign_pool, sign_pitch,
                                 d_temp_pool, temp_pitch, lut, exec_threshold, batch, (cudaStream_t)stream,
                                 cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost))
}

int cudil_sign_randomized(int mode, uint8_t *sig, size_t sig_pitch, size_t *siglen, const uint8_t *m, size_t m_pitch,
                          size_t mlen, const uint8_t *sk, const uint8_t *rhoprime, size_t rhoprime_pitch,
                          uint8_t *d_sign_pool, size_t sign_pitch, uint8_t *d_temp_pool, size_t temp_pitch,
                          cudil_task_lut *lut, size_t exec_threshold, size_t batch, void *stream) {
    if (!rhoprime && batch) return CUDIL_ERR_INVALID;
    CUDIL_DISPATCH(mode, I::sign(sig, sig_pitch, siglen, m, m_pitch, mlen, sk, I::PM::SK_BYTES, d_sign_pool, sign_pitch,
                                 d_temp_pool, temp_pitch, lut, exec_threshold, batch, (cudaStream_t)stream,
                                 cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost, nullptr, rhoprime, rhoprime_pitch))
}

int cudil_sign_dev_randomized(int mode, uint8_t *d_sig, size_t sig_pitch, const uint8_t *d_m, size_t m_pitch,
                              size_t mlen, const uint8_t *d_sk, const uint8_t *d_rhoprime, size_t rhoprime_pitch,
                              uint8_t *d_sign_pool, size_t sign_pitch, uint8_t *d_temp_pool, size_t temp_pitch,
                              cudil_task_lut *lut, size_t exec_threshold, size_t batch, void *stream) {
    if (!d_rhoprime && batch) return CUDIL_ERR_INVALID;
    CUDIL_DISPATCH(mode, I::sign(d_sig, sig_pitch, nullptr, d_m, m_pitch, mlen, d_sk, I::PM::SK_BYTES, d_sign_pool,
                                 sign_pitch, d_temp_pool, temp_pitch, lut, exec_threshold, batch, (cudaStream_t)stream,
                                 cudaMemcpyDeviceToDevice, cudaMemcpyDeviceToDevice, nullptr, d_rhoprime,
                                 rhoprime_pitch))
}

int cudil_sign_dev(int mode, uint8_t *d_sig, size_t sig_pitch, const uint8_t *d_m, size_t m_pitch, size_t mlen,
                   const uint8_t *d_sk, uint8_t *d_sign_pool, size_t sign_pitch, uint8_t *d_temp_pool, size_t temp_pitch,
                   cudil_task_lut *lut, size_t exec_threshold, size_t batch, void *stream) {
    CUDIL_DISPATCH(mode, I::sign(d_sig, sig_pitch, nullptr, d_m, m_pitch, mlen, d_sk, I::PM::SK_BYTES, d_sign_pool,
                                 sign_pitch, d_temp_pool, temp_pitch, lut, exec_threshold, batch, (cudaStream_t)stream,
                                 cudaMemcpyDeviceToDevice, cudaMemcpyDeviceToDevice))
}

int cudil_verify(int mode, int *ret, const uint8_t *sig, size_t sig_pitch, size_t siglen, const uint8_t *m,
                 size_t m_pitch, size_t mlen, const uint8_t *pk, uint8_t *d_pool, size_t pitch, size_t batch,
                 void *stream) {
    CUDIL_DISPATCH(mode, I::verify(ret, sig, sig_pitch, siglen, m, m_pitch, mlen, pk, I::PM::PK_BYTES, d_pool, pitch,
                                   batch, (cudaStream_t)stream, cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost))
}

int cudil_crypto_sign(int mode, uint8_t *sm, size_t sm_pitch, size_t *smlen, const uint8_t *m, size_t m_pitch,
                      size_t mlen, const uint8_t *sk, uint8_t *d_sign_pool, size_t sign_pitch, uint8_t *d_temp_pool,
                      size_t temp_pitch, cudil_task_lut *lut, size_t exec_threshold, size_t batch, void *stream) {
    cudil_params p;
    if (cudil_get_params(mode, &p) != CUDIL_OK) return CUDIL_ERR_INVALID;
    const size_t sb = (size_t)p.sig_bytes;
    if (smlen) *smlen = sb + mlen;
    if (batch == 0) return CUDIL_OK;
    if (!sm || (mlen && !m) || sm_pitch < sb + mlen) return CUDIL_ERR_INVALID;
    // message behind the signature slot first (memmove: m may already sit inside sm), then sign
    // with the message read from its place in sm and the signature written in front of it
    for (size_t i = 0; i < batch && mlen; ++i) std::memmove(sm + i * sm_pitch + sb, m + i * m_pitch, mlen);
    return cudil_sign(mode, sm, sm_pitch, nullptr, sm + sb, sm_pitch, mlen, sk, d_sign_pool, sign_pitch, d_temp_pool,
                      temp_pitch, lut, exec_threshold, batch, stream);
}

int cudil_crypto_sign_open(int mode, uint8_t *m, size_t m_pitch, size_t *mlen, int *ret, const uint8_t *sm,
                           size_t sm_pitch, size_t smlen, const uint8_t *pk, uint8_t *d_verify_pool, size_t verify_pitch,
                           size_t batch, void *stream) {
    cudil_params p;
    if (cudil_get_params(mode, &p) != CUDIL_OK) return CUDIL_ERR_INVALID;
    const size_t sb = (size_t)p.sig_bytes;
    if (batch == 0) return CUDIL_OK;
    if (!ret || !m || !sm || !mlen) return CUDIL_ERR_INVALID;
    if (smlen < sb) {
        *mlen = 0;
        for (size_t i = 0; i < batch; ++i) ret[i] = -1;
        return CUDIL_OK;
    }
    const size_t ml = smlen - sb;
    if (sm_pitch < smlen || (ml && m_pitch < ml)) return CUDIL_ERR_INVALID;
    int rc = cudil_verify(mode, ret, sm, sm_pitch, sb, sm + sb, sm_pitch, ml, pk, d_verify_pool, verify_pitch, batch,
                          stream);
    if (rc) return rc;
    // the messages are released only for valid signatures: wait for the results
    if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess)
        return cudil::cudil_record_cuda_error(cudaGetLastError(), __FILE__, __LINE__);
    *mlen = ml;
    for (size_t i = 0; i < batch && ml; ++i) {
        if (ret[i] == 0)
            std::memmove(m + i * m_pitch, sm + i * sm_pitch + sb, ml);
        else
            std::memset(m + i * m_pitch, 0, ml);
    }
    return CUDIL_OK;
}

int cudil_verify_dev(int mode, int *d_ret, const uint8_t *d_sig, size_t sig_pitch, size_t siglen, const uint8_t *d_m,
                     size_t m_pitch, size_t mlen, const uint8_t *d_pk, uint8_t *d_pool, size_t pitch, size_t batch,
                     void *stream) {
    CUDIL_DISPATCH(mode, I::verify(d_ret, d_sig, sig_pitch, siglen, d_m, m_pitch, mlen, d_pk, I::PM::PK_BYTES, d_pool,
                                   pitch, batch, (cudaStream_t)stream, cudaMemcpyDeviceToDevice, cudaMemcpyDeviceToDevice))
}

int cudil_sign_dev_varlen(int mode, uint8_t *d_sig, size_t sig_pitch, const uint8_t *d_m, size_t m_pitch,
                          const uint32_t *d_mlens, size_t max_mlen, const uint8_t *d_sk, uint8_t *d_sign_pool,
                          size_t sign_pitch, uint8_t *d_temp_pool, size_t temp_pitch, cudil_task_lut *lut,
                          size_t exec_threshold, size_t batch, void *stream) {
    if (!d_mlens) return CUDIL_ERR_INVALID;
    CUDIL_DISPATCH(mode, I::sign(d_sig, sig_pitch, nullptr, d_m, m_pitch, max_mlen, d_sk, I::PM::SK_BYTES, d_sign_pool,
                                 sign_pitch, d_temp_pool, temp_pitch, lut, exec_threshold, batch, (cudaStream_t)stream,
                                 cudaMemcpyDeviceToDevice, cudaMemcpyDeviceToDevice, d_mlens))
}

int cudil_verify_dev_varlen(int mode, int *d_ret, const uint8_t *d_sig, size_t sig_pitch, size_t siglen,
                            const uint8_t *d_m, size_t m_pitch, const uint32_t *d_mlens, size_t max_mlen,
                            const uint8_t *d_pk, uint8_t *d_pool, size_t pitch, size_t batch, void *stream) {
    if (!d_mlens) return CUDIL_ERR_INVALID;
    CUDIL_DISPATCH(mode, I::verify(d_ret, d_sig, sig_pitch, siglen, d_m, m_pitch, max_mlen, d_pk, I::PM::PK_BYTES, d_pool,
                                   pitch, batch, (cudaStream_t)stream, cudaMemcpyDeviceToDevice, cudaMemcpyDeviceToDevice,
                                   d_mlens))
}

}  // extern "C"

namespace {
template <int MODE>
int sig_check_impl(int *d_status, const uint8_t *d_sig, size_t sig_pitch, size_t n, cudaStream_t st) {
    using namespace cudil;
    if (n == 0) return CUDIL_OK;
    if (!d_status || !d_sig || sig_pitch < (size_t)P<MODE>::SIG_BYTES || n > (size_t)INT_MAX / 32) return CUDIL_ERR_INVALID;
    CUDIL_LAUNCH(KID_SIG_CHECK, st, k_sig_check<MODE><<<blocks_for(n * 32), kBlock, 0, st>>>(d_status, d_sig, sig_pitch, (int)n));
    CUDIL_CK_LAUNCH();
    return CUDIL_OK;
}
template <int MODE>
int sk_check_impl(int *d_status, const uint8_t *d_sk, size_t n, cudaStream_t st) {
    using namespace cudil;
    if (n == 0) return CUDIL_OK;
    if (!d_status || !d_sk || n > (size_t)INT_MAX / 32) return CUDIL_ERR_INVALID;
    CUDIL_LAUNCH(KID_SK_CHECK, st, k_sk_check<MODE><<<blocks_for(n * 32), kBlock, 0, st>>>(d_status, d_sk, (int)n));
    CUDIL_CK_LAUNCH();
    return CUDIL_OK;
}
}  // namespace

extern "C" {

int cudil_sig_check(int mode, int *d_status, const uint8_t *d_sig, size_t sig_pitch, size_t batch, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    switch (mode) {
        case 2: return sig_check_impl<2>(d_status, d_sig, sig_pitch, batch, st);
        case 3: return sig_check_impl<3>(d_status, d_sig, sig_pitch, batch, st);
        case 5: return sig_check_impl<5>(d_status, d_sig, sig_pitch, batch, st);
        default: return CUDIL_ERR_INVALID;
    }
}

int cudil_sk_check(int mode, int *d_status, const uint8_t *d_sk, size_t batch, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    switch (mode) {
        case 2: return sk_check_impl<2>(d_status, d_sk, batch, st);
        case 3: return sk_check_impl<3>(d_status, d_sk, batch, st);
        case 5: return sk_check_impl<5>(d_status, d_sk, batch, st);
        default: return CUDIL_ERR_INVALID;
    }
}

int cudil_ntt_mul(const int32_t *d_a, const int32_t *d_b, int32_t *d_out, size_t npolys, void *stream) {
    if (npolys == 0) return CUDIL_OK;
    if (!d_a || !d_b || !d_out) return CUDIL_ERR_INVALID;
    const size_t threads = npolys * 16;
    cudaStream_t st = (cudaStream_t)stream;
    // a few resident blocks per SM, each group looping over its share of the batch
    static int blocks = 0;
    if (!blocks) {
        int dev = 0, sms = 0, per_sm = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ntt_mul, kBlock, 0) != cudaSuccess || per_sm < 1)
            return cudil::cudil_record_cuda_error(cudaGetLastError(), __FILE__, __LINE__);
        blocks = sms * per_sm;
    }
    const size_t need = (threads + kBlock - 1) / kBlock;
    const unsigned grid = (unsigned)(need < (size_t)blocks ? need : (size_t)blocks);
    CUDIL_LAUNCH(KID_NTT_MUL, st, k_ntt_mul<<<grid, kBlock, 0, st>>>(d_a, d_b, d_out, (long long)npolys));
    return cudaGetLastError() == cudaSuccess ? CUDIL_OK : CUDIL_ERR_CUDA;
}

int cudil_derive_rhoprime(uint8_t *d_rhoprime, size_t rhoprime_pitch, const uint8_t *seed, unsigned long long counter,
                          size_t n, void *stream) {
    if (n == 0) return CUDIL_OK;
    if (!d_rhoprime || !seed || rhoprime_pitch < 64 || n > (size_t)LLONG_MAX / rhoprime_pitch) return CUDIL_ERR_INVALID;
    Seed32 s;
    std::memcpy(s.w, seed, sizeof s.w);
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned blocks = (unsigned)((n + kBlock - 1) / kBlock);
    CUDIL_LAUNCH(KID_DERIVE_RHOP, st,
                 k_derive_rhoprime<<<blocks, kBlock, 0, st>>>(d_rhoprime, rhoprime_pitch, s, counter, (long long)n));
    return cudaGetLastError() == cudaSuccess ? CUDIL_OK : CUDIL_ERR_CUDA;
}

int cudil_bounds_check_status(unsigned *error, int reset) {
    if (!error) return CUDIL_ERR_INVALID;
    *error = 0;
    if (!kBoundsChecked) return CUDIL_ERR_INVALID;
    cudaError_t (*const words[])(unsigned *, bool) = {bounds_status_mode2, bounds_status_mode3, bounds_status_mode5,
                                                      bounds_status_here};
    for (auto fn : words) {
        unsigned v = 0;
        const cudaError_t e = fn(&v, reset != 0);
        if (e != cudaSuccess) return cudil_record_cuda_error(e, __FILE__, __LINE__);
        if (!*error) *error = v;
    }
    return CUDIL_OK;
}

int cudil_alu_peak(uint32_t *d_out, int blocks, int iters, void *stream, double *ops_per_launch) {
    if (!d_out || blocks <= 0 || iters <= 0) return CUDIL_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    CUDIL_LAUNCH(KID_ALU_PEAK, st, k_alu_peak<<<blocks, 256, 0, st>>>(d_out, iters));
    if (ops_per_launch) *ops_per_launch = (double)blocks * 256.0 * iters * 8.0 * 4.0;
    return cudaGetLastError() == cudaSuccess ? CUDIL_OK : CUDIL_ERR_CUDA;
}

unsigned long long cudil_launch_count(void) { return Profiler::get().launches.load(); }

void cudil_kernel_timing(int enable) {
    Profiler::get().collect();
    Profiler::get().timing.store(enable ? 1 : 0);
}

int cudil_kernel_count(void) { return KID_COUNT; }

const char *cudil_kernel_name(int id) { return kernel_name(id); }

int cudil_kernel_stats(int id, double *total_ms, unsigned long long *launches) {
    if (id < 0 || id >= KID_COUNT) return CUDIL_ERR_INVALID;
    Profiler &p = Profiler::get();
    p.collect();
    if (total_ms) *total_ms = p.total_ms[id];
    if (launches) *launches = p.count[id];
    return CUDIL_OK;
}

void cudil_kernel_stats_reset(void) { Profiler::get().reset(); }

}  // extern "C"
