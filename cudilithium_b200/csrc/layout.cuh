// Where each kernel keeps its per-item data inside the caller-allocated pitched pools.
//
// The drop-in entry points receive the same pools as the reference (src/api.cu:26-515) and the
// caller sizes their rows with the reference's formulas (tests/test_vectors.cu:62-166); every
// layout below fits inside that row budget (checked by static_asserts / host checks), so a caller
// that sized pools for the reference can switch without changing its allocations.
#pragma once

#include <cstddef>

#include "params.cuh"

namespace cudil {

template <int MODE>
struct Layout {
    using PM = P<MODE>;
    static constexpr int K = PM::K, L = PM::L;
    static constexpr size_t POLY = N * sizeof(int32_t);

    // ---- reference row budgets (bytes per item) ----
    static constexpr size_t ref_keypair_row() { return align256(PM::PK_BYTES) + align256(PM::SK_BYTES) + K * POLY; }
    static constexpr size_t ref_sign_row(size_t mlen) {
        return align256(PM::SIG_BYTES) + align256(PM::SK_BYTES) + align256(SEEDBYTES) + align256(SEEDBYTES + mlen) +
               align256(SEEDBYTES + CRHBYTES + PM::W1PACKED_BYTES) + align256(CRHBYTES) +
               (size_t)(K * L + 3 * L + 4 * K + 1) * POLY;
    }
    static constexpr size_t ref_sign_temp_row() {
        return align256(PM::SIG_BYTES) + align256(CRHBYTES + PM::W1PACKED_BYTES) + (size_t)(2 * L + 3 * K) * POLY;
    }
    static constexpr size_t ref_verify_row(size_t mlen) {
        return align256(PM::SIG_BYTES) + align256(PM::PK_BYTES) + align256(SEEDBYTES + mlen) +
               align256(CRHBYTES + PM::W1PACKED_BYTES) + align256(SEEDBYTES) + (size_t)(K * L + L + 3 * K + 1) * POLY +
               sizeof(int);
    }

    // ---- keypair row: pk | sk | t_hat accumulators (K polys, zeroed before use) ----
    static constexpr size_t KP_PK = 0;
    static constexpr size_t KP_SK = align256(PM::PK_BYTES);
    static constexpr size_t KP_TACC = KP_SK + align256(PM::SK_BYTES);
    static constexpr size_t KP_END = KP_TACC + K * POLY;
    // rho' is parked in pk's t1 area until t1 is packed.
    static constexpr size_t KP_RHOP = KP_PK + SEEDBYTES;

    // ---- sign row: sig | sk | mu,rho' | m | A_hat | s1_hat | s2_hat | t0_hat ----
    static constexpr size_t SG_SIG = 0;
    static constexpr size_t SG_SK = align256(PM::SIG_BYTES);
    static constexpr size_t SG_MU = SG_SK + align256(PM::SK_BYTES);
    static constexpr size_t SG_RHOP = SG_MU + CRHBYTES;
    static constexpr size_t SG_MSG = SG_MU + 256;
    static constexpr size_t sg_mat(size_t mlen) { return SG_MSG + align256(mlen); }
    static constexpr size_t sg_s1(size_t mlen) { return sg_mat(mlen) + (size_t)K * L * POLY; }
    static constexpr size_t sg_s2(size_t mlen) { return sg_s1(mlen) + (size_t)L * POLY; }
    static constexpr size_t sg_t0(size_t mlen) { return sg_s2(mlen) + (size_t)K * POLY; }
    static constexpr size_t sg_end(size_t mlen) { return sg_t0(mlen) + (size_t)K * POLY; }

    // ---- sign temp row (one per speculative attempt): sig | w1 packed | y packed | w0 | c masks ----
    static constexpr size_t TP_SIG = 0;
    static constexpr size_t TP_W1P = align256(PM::SIG_BYTES);
    static constexpr size_t TP_Y = TP_W1P + align256(PM::W1PACKED_BYTES);
    static constexpr size_t TP_W0 = TP_Y + align256((size_t)L * PM::POLYZ_PACKED);
    static constexpr size_t TP_CMASK = TP_W0 + (size_t)K * POLY;
    static constexpr size_t TP_END = TP_CMASK + 64;

    // ---- verify row: sig | pk | tr'||m | mu||w1' | aux (c masks, status, ret) | A_hat ----
    static constexpr size_t VF_SIG = 0;
    static constexpr size_t VF_PK = align256(PM::SIG_BYTES);
    static constexpr size_t VF_TRM = VF_PK + align256(PM::PK_BYTES);
    static constexpr size_t vf_mu(size_t mlen) { return VF_TRM + align256(SEEDBYTES + mlen); }
    static constexpr size_t vf_aux(size_t mlen) { return vf_mu(mlen) + align256(CRHBYTES + PM::W1PACKED_BYTES); }
    // aux: [0,64) c masks, [64,68) status (0 = ok so far), [68,72) ret
    static constexpr size_t vf_mat(size_t mlen) { return vf_aux(mlen) + 256; }
    static constexpr size_t vf_end(size_t mlen) { return vf_mat(mlen) + (size_t)K * L * POLY; }

    static_assert(KP_END <= ref_keypair_row(), "keypair row exceeds the reference budget");
    static_assert(TP_END <= ref_sign_temp_row(), "temp row exceeds the reference budget");
    static_assert(sg_end(32) <= ref_sign_row(32), "sign row exceeds the reference budget");
    static_assert(sg_end(65536) <= ref_sign_row(65536), "sign row exceeds the reference budget");
    static_assert(vf_end(32) <= ref_verify_row(32), "verify row exceeds the reference budget");
    static_assert(vf_end(65536) <= ref_verify_row(65536), "verify row exceeds the reference budget");
};

}  // namespace cudil
