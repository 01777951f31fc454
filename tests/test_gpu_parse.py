"""Batched well-formedness checks (cudil_sig_check / cudil_sk_check) against the oracle's
restatement of the reference's hint-encoding and z checks (src/verify.cu:51-121) and of the eta
encoding (needs a B200)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MODES = [2, 3, 5]


def tampered_signatures(oracle, mode, sig, rng):
    """Valid signatures plus malformed variants of each kind the checks distinguish."""
    p = oracle.params(mode)
    h0 = 32 + p.l * p.polyz_packed
    out = [sig.copy() for _ in range(8)]
    out[1][:, h0 + p.omega + p.k - 1] = p.omega + 1          # end count above omega
    out[2][:, h0 + p.omega] = 5                              # first poly claims positions ...
    out[2][:, h0 + 0: h0 + 5] = [9, 3, 4, 5, 6]              # ... not strictly increasing
    out[2][:, h0 + p.omega + 1: h0 + p.omega + p.k] = np.maximum(out[2][:, h0 + p.omega + 1: h0 + p.omega + p.k], 5)
    out[3][:, h0 + p.omega - 1] = 7                          # unused slot not zero (normally)
    out[4][:, h0 + p.omega + 1] = 0                          # counts decreasing (poly 1 < poly 0)
    out[4][:, h0 + p.omega] = np.maximum(out[4][:, h0 + p.omega], 1)
    out[5][:, 32: 35] = 0                                    # z0 = gamma1 - 0 = gamma1: out of range
    for i in range(out[6].shape[0]):                         # random byte flips anywhere
        out[6][i, int(rng.integers(0, p.sig_bytes))] ^= np.uint8(1 << int(rng.integers(0, 8)))
    out[7] = rng.integers(0, 256, sig.shape, dtype=np.uint8)  # garbage
    return np.concatenate(out)


@pytest.mark.parametrize("mode", MODES)
def test_sig_check_matches_oracle(cuda_ok, oracle, mode):
    import cudilithium_b200 as cd
    rng = np.random.default_rng(800 + mode)
    n = 24
    pk, sk = oracle.keypair_batch(mode, n, rand_index=8200 + mode)
    m = oracle.messages_from_ctr(n, 32)
    sig = oracle.sign_batch(mode, m, sk)
    allsig = tampered_signatures(oracle, mode, sig, rng)
    want = oracle.sig_check(mode, allsig)
    got = cd.Dilithium(mode).sig_check(allsig)
    assert np.array_equal(got, want)
    assert np.all(want[:n] == 0)
    assert (want & 1).any() and (want & 2).any()
    # every signature the check flags is rejected by verification
    mm = np.tile(m, (allsig.shape[0] // n, 1))
    pkk = np.tile(pk, (allsig.shape[0] // n, 1))
    ret = oracle.verify_batch(mode, allsig, mm, pkk)
    assert np.all(ret[want != 0] == -1)


@pytest.mark.parametrize("mode", MODES)
def test_sig_check_pitched_rows(cuda_ok, oracle, mode):
    import cudilithium_b200 as cd
    p = oracle.params(mode)
    pk, sk = oracle.keypair_batch(mode, 5, rand_index=8300 + mode)
    sig = oracle.sign_batch(mode, oracle.messages_from_ctr(5, 32), sk)
    sig[2, 32 + p.l * p.polyz_packed + p.omega + p.k - 1] = 255
    pitch = p.sig_bytes + 13
    rows = np.zeros((5, pitch), np.uint8)
    rows[:, : p.sig_bytes] = sig
    got = cd.Dilithium(mode).sig_check(rows, sig_pitch=pitch)
    assert np.array_equal(got, oracle.sig_check(mode, sig))
    assert got[2] & 1 and got[[0, 1, 3, 4]].sum() == 0


@pytest.mark.parametrize("mode", MODES)
def test_sk_check_matches_oracle(cuda_ok, oracle, mode):
    import cudilithium_b200 as cd
    rng = np.random.default_rng(900 + mode)
    p = oracle.params(mode)
    n = 30
    pk, sk = oracle.keypair_batch(mode, n, rand_index=9100 + mode)
    bad = sk.copy()
    # random bytes in the s1 / s2 region of every odd key (out-of-range fields are then likely)
    s_end = 96 + (p.l + p.k) * p.polyeta_packed
    for i in range(1, n, 2):
        j = int(rng.integers(96, s_end))
        bad[i, j] = 0xFF
    allsk = np.concatenate([sk, bad])
    want = oracle.sk_check(mode, allsk)
    got = cd.Dilithium(mode).sk_check(allsk)
    assert np.array_equal(got, want)
    assert np.all(want[:n] == 0) and want[n + 1::2].all()


def test_check_invalid_arguments(cuda_ok):
    import ctypes

    from cudilithium_b200._lib import CUDIL_ERR_INVALID, CUDIL_OK, lib
    assert lib.cudil_sig_check(4, None, None, 0, 1, None) == CUDIL_ERR_INVALID
    assert lib.cudil_sig_check(2, None, None, 2420, 0, None) == CUDIL_OK
    assert lib.cudil_sig_check(2, ctypes.c_void_p(16), ctypes.c_void_p(16), 100, 1, None) == CUDIL_ERR_INVALID
    assert lib.cudil_sk_check(2, None, None, 3, None) == CUDIL_ERR_INVALID
