// A caller of the reference's C++ API, built against include/api.cuh and linked with
// libcudilithium_b200.so: the known-answer flow of the reference's test (keypair -> sign -> verify
// of a batch, pools sized with the reference's formulas and macros, exec_threshold 2048).
//
//   kat_shim <dir> <n> <mlen>
// reads <dir>/m.bin (n * mlen bytes) and writes pk.bin, sk.bin, sig.bin, ret.bin there.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "api.cuh"

static bool read_file(const char *dir, const char *name, void *p, size_t n) {
    char path[4096];
    std::snprintf(path, sizeof path, "%s/%s", dir, name);
    FILE *f = std::fopen(path, "rb");
    if (!f) return false;
    const bool ok = std::fread(p, 1, n, f) == n;
    std::fclose(f);
    return ok;
}

static bool write_file(const char *dir, const char *name, const void *p, size_t n) {
    char path[4096];
    std::snprintf(path, sizeof path, "%s/%s", dir, name);
    FILE *f = std::fopen(path, "wb");
    if (!f) return false;
    const bool ok = std::fwrite(p, 1, n, f) == n;
    std::fclose(f);
    return ok;
}

int main(int argc, char **argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s <dir> <n> <mlen>\n", argv[0]);
        return 2;
    }
    const char *dir = argv[1];
    const size_t n = std::strtoull(argv[2], nullptr, 10), mlen = std::strtoull(argv[3], nullptr, 10);

    uint8_t *h_pk, *h_sk, *h_m, *h_sig;
    int *h_ret;
    cudaMallocHost(&h_pk, n * CRYPTO_PUBLICKEYBYTES);
    cudaMallocHost(&h_sk, n * CRYPTO_SECRETKEYBYTES);
    cudaMallocHost(&h_m, n * mlen + 1);
    cudaMallocHost(&h_sig, n * CRYPTO_BYTES);
    cudaMallocHost(&h_ret, n * sizeof(int));
    if (!read_file(dir, "m.bin", h_m, n * mlen)) return 3;

    // key generation pool: pk, sk and K polynomials per key
    const size_t kp_row = ALIGN_TO_256_BYTES(CRYPTO_PUBLICKEYBYTES) + ALIGN_TO_256_BYTES(CRYPTO_SECRETKEYBYTES) +
                          DILITHIUM_K * DILITHIUM_N * sizeof(int32_t);
    uint8_t *d_kp;
    size_t kp_pitch;
    if (cudaMallocPitch(&d_kp, &kp_pitch, kp_row, n) != cudaSuccess) return 4;
    if (crypto_sign_keypair(h_pk, h_sk, d_kp, kp_pitch, n) != 0) return 5;
    cudaDeviceSynchronize();
    cudaFree(d_kp);

    // signing pools: per message and per exec slot
    const size_t sign_row = ALIGN_TO_256_BYTES(CRYPTO_BYTES) + ALIGN_TO_256_BYTES(CRYPTO_SECRETKEYBYTES) +
                            ALIGN_TO_256_BYTES(SEEDBYTES) + ALIGN_TO_256_BYTES(SEEDBYTES + mlen) +
                            ALIGN_TO_256_BYTES(SEEDBYTES + CRHBYTES + DILITHIUM_K * POLYW1_PACKEDBYTES) +
                            ALIGN_TO_256_BYTES(CRHBYTES) +
                            (DILITHIUM_K * DILITHIUM_L + 3 * DILITHIUM_L + 4 * DILITHIUM_K + 1) * DILITHIUM_N *
                                sizeof(int32_t);
    const size_t exec_threshold = 2048;
    const size_t temp_row = ALIGN_TO_256_BYTES(CRYPTO_BYTES) +
                            ALIGN_TO_256_BYTES(CRHBYTES + DILITHIUM_K * POLYW1_PACKEDBYTES) +
                            (2 * DILITHIUM_L + 3 * DILITHIUM_K) * DILITHIUM_N * sizeof(int32_t);
    uint8_t *d_sign, *d_temp;
    size_t sign_pitch, temp_pitch;
    if (cudaMallocPitch(&d_sign, &sign_pitch, sign_row, n) != cudaSuccess ||
        cudaMallocPitch(&d_temp, &temp_pitch, temp_row, exec_threshold) != cudaSuccess)
        return 4;
    task_lut lut{};
    lut.sign_lut.resize(n);
    cudaMallocHost(&lut.h_exec_lut, sizeof(uint32_t) * exec_threshold);
    cudaMallocHost(&lut.h_done_lut, sizeof(uint8_t) * exec_threshold);
    cudaMallocHost(&lut.h_copy_lut, sizeof(copy_lut_element) * exec_threshold);
    cudaMalloc(&lut.d_exec_lut, sizeof(uint32_t) * exec_threshold);
    cudaMalloc(&lut.d_done_lut, sizeof(uint8_t) * exec_threshold);
    cudaMalloc(&lut.d_copy_lut, sizeof(copy_lut_element) * exec_threshold);
    size_t siglen = 0;
    if (crypto_sign_signature(h_sig, CRYPTO_BYTES, &siglen, h_m, mlen, mlen, h_sk, d_sign, sign_pitch, d_temp,
                              temp_pitch, lut, exec_threshold, n) != 0)
        return 6;
    cudaDeviceSynchronize();
    if (siglen != CRYPTO_BYTES) return 7;

    // verification pool: signature, pk, message, hashes and the expanded matrix per item
    const size_t verify_row = ALIGN_TO_256_BYTES(CRYPTO_BYTES) + ALIGN_TO_256_BYTES(CRYPTO_PUBLICKEYBYTES) +
                              ALIGN_TO_256_BYTES(SEEDBYTES + mlen) +
                              ALIGN_TO_256_BYTES(CRHBYTES + DILITHIUM_K * POLYW1_PACKEDBYTES) +
                              ALIGN_TO_256_BYTES(SEEDBYTES) +
                              (DILITHIUM_K * DILITHIUM_L + DILITHIUM_L + 3 * DILITHIUM_K + 1) * DILITHIUM_N *
                                  sizeof(int32_t) +
                              sizeof(int);
    uint8_t *d_verify;
    size_t verify_pitch;
    if (cudaMallocPitch(&d_verify, &verify_pitch, verify_row, n) != cudaSuccess) return 4;
    crypto_sign_verify(h_ret, h_sig, CRYPTO_BYTES, CRYPTO_BYTES, h_m, mlen, mlen, h_pk, d_verify, verify_pitch, n);
    cudaDeviceSynchronize();
    if (cudaGetLastError() != cudaSuccess) return 8;

    const bool ok = write_file(dir, "pk.bin", h_pk, n * CRYPTO_PUBLICKEYBYTES) &&
                    write_file(dir, "sk.bin", h_sk, n * CRYPTO_SECRETKEYBYTES) &&
                    write_file(dir, "sig.bin", h_sig, n * CRYPTO_BYTES) && write_file(dir, "ret.bin", h_ret, n * sizeof(int));
    std::printf("mode %d: %zu items, pk %d sk %d sig %d bytes\n", DILITHIUM_MODE, n, CRYPTO_PUBLICKEYBYTES,
                CRYPTO_SECRETKEYBYTES, CRYPTO_BYTES);
    return ok ? 0 : 9;
}
