// Dilithium round-3 (v3.1) parameter sets as compile-time types, so that one binary carries
// all three sets (the reference selects one per library with DILITHIUM_MODE,
// include/params.h:14-45 of the reference).
#pragma once

#include <cstddef>
#include <cstdint>

namespace cudil {

constexpr int N = 256;
constexpr int Q = 8380417;
constexpr int QINV = 58728449;  // q^-1 mod 2^32
constexpr int D = 13;
constexpr int SEEDBYTES = 32;
constexpr int CRHBYTES = 64;
constexpr int SHAKE128_RATE = 168;
constexpr int SHAKE256_RATE = 136;
constexpr int POLYT1_PACKED = 320;
constexpr int POLYT0_PACKED = 416;

__host__ __device__ constexpr size_t align256(size_t x) { return (x + 255) / 256 * 256; }

template <int MODE>
struct Params;

template <>
struct Params<2> {
    static constexpr int K = 4, L = 4, ETA = 2, TAU = 39, BETA = 78, OMEGA = 80;
    static constexpr int GAMMA1 = 1 << 17, GAMMA2 = (Q - 1) / 88;
};
template <>
struct Params<3> {
    static constexpr int K = 6, L = 5, ETA = 4, TAU = 49, BETA = 196, OMEGA = 55;
    static constexpr int GAMMA1 = 1 << 19, GAMMA2 = (Q - 1) / 32;
};
template <>
struct Params<5> {
    static constexpr int K = 8, L = 7, ETA = 2, TAU = 60, BETA = 120, OMEGA = 75;
    static constexpr int GAMMA1 = 1 << 19, GAMMA2 = (Q - 1) / 32;
};

// Sizes derived from a parameter set (include/params.h:47-73 of the reference).
template <int MODE>
struct P : Params<MODE> {
    using B = Params<MODE>;
    static constexpr int Z_BITS = (B::GAMMA1 == (1 << 17)) ? 18 : 20;
    static constexpr int W1_BITS = (B::GAMMA2 == (Q - 1) / 88) ? 6 : 4;
    static constexpr int W1_MAX = (B::GAMMA2 == (Q - 1) / 88) ? 43 : 15;
    static constexpr int ETA_BITS = (B::ETA == 2) ? 3 : 4;
    static constexpr int POLYZ_PACKED = 32 * Z_BITS;        // 576 / 640
    static constexpr int POLYW1_PACKED = 32 * W1_BITS;      // 192 / 128
    static constexpr int POLYETA_PACKED = 32 * ETA_BITS;    // 96 / 128
    static constexpr int POLYVECH_PACKED = B::OMEGA + B::K;
    static constexpr int PK_BYTES = SEEDBYTES + B::K * POLYT1_PACKED;
    static constexpr int SK_BYTES = 3 * SEEDBYTES + (B::L + B::K) * POLYETA_PACKED + B::K * POLYT0_PACKED;
    static constexpr int SIG_BYTES = SEEDBYTES + B::L * POLYZ_PACKED + POLYVECH_PACKED;
    static constexpr int W1PACKED_BYTES = B::K * POLYW1_PACKED;
    // SHAKE256 blocks of ExpandMask (5 for every set) and ExpandS (first batch).
    static constexpr int MASK_BLOCKS = (POLYZ_PACKED + SHAKE256_RATE - 1) / SHAKE256_RATE;
    // offsets inside sk
    static constexpr int SK_RHO = 0, SK_KEY = 32, SK_TR = 64, SK_S1 = 96;
    static constexpr int SK_S2 = SK_S1 + B::L * POLYETA_PACKED;
    static constexpr int SK_T0 = SK_S2 + B::K * POLYETA_PACKED;
    // offsets inside sig
    static constexpr int SIG_Z = SEEDBYTES;
    static constexpr int SIG_H = SEEDBYTES + B::L * POLYZ_PACKED;
};

}  // namespace cudil
