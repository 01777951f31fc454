"""CUDA path vs the CPU oracle and the reference's golden digests (needs a B200).

Every call goes through the C ABI (libcudilithium_b200.so via ctypes); the oracle is only the
checker.  Results must be bit-exact.
"""
import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MODES = [2, 3, 5]


def messages(n, mlen):
    return np.stack([np.frombuffer(hashlib.shake_128((2 * i).to_bytes(8, "little")).digest(mlen), dtype=np.uint8)
                     for i in range(n)]) if mlen else np.zeros((n, 0), np.uint8)


@pytest.fixture(scope="module")
def dil(cuda_ok):
    from cudilithium_b200 import Dilithium
    return {m: Dilithium(m) for m in MODES}


@pytest.mark.parametrize("mode", MODES)
def test_gpu_tvecs_digest_matches_reference(dil, oracle, golden_digests, mode):
    """The full known-answer test of the reference (10000 keys/signatures per mode) on the GPU."""
    n = golden_digests["nvectors"]
    d = dil[mode]
    m = messages(n, 32)
    pk, sk = d.keypair(n, rand_index=0)
    sig = d.sign(m, sk, exec_threshold=2048)
    ret = d.verify(sig, m, pk)
    assert np.all(ret == 0)
    data = oracle.tvecs_from_outputs(m, pk, sk, sig, ret)
    assert hashlib.sha256(data).hexdigest() == golden_digests["sha256"][str(mode)]


@pytest.mark.parametrize("mode", MODES)
def test_keypair_matches_oracle(dil, oracle, mode):
    for n, ri in [(1, 0), (37, 12345), (300, 7)]:
        pk, sk = dil[mode].keypair(n, rand_index=ri)
        opk, osk = oracle.keypair_batch(mode, n, rand_index=ri)
        assert np.array_equal(pk, opk)
        assert np.array_equal(sk, osk)


@pytest.mark.parametrize("mode", MODES)
def test_keypair_from_seed_matches_oracle(dil, oracle, mode):
    rng = np.random.default_rng(mode)
    seeds = rng.integers(0, 256, (45, 32), dtype=np.uint8)
    pk, sk = dil[mode].keypair(45, seeds=seeds)
    opk, osk = oracle.keypair_seeds(mode, seeds)
    assert np.array_equal(pk, opk) and np.array_equal(sk, osk)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("threshold", [1, 5, 64, 3000])
def test_sign_matches_oracle_any_exec_threshold(dil, oracle, mode, threshold):
    """Smallest-accepted-nonce semantics do not depend on how attempts are scheduled."""
    n = 40
    pk, sk = oracle.keypair_batch(mode, n, rand_index=99)
    m = messages(n, 59)
    sig, lut = dil[mode].sign(m, sk, exec_threshold=threshold, return_lut=True)
    osig, att = oracle.sign_batch(mode, m, sk, return_attempts=True)
    assert np.array_equal(sig, osig)
    assert np.all(dil[mode].verify(sig, m, pk) == 0)
    # every item was tried at least up to its winning nonce
    assert np.all(lut.nonces() >= att)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("mlen", [0, 1, 7, 8, 103, 104, 135, 136, 137, 271, 1000, 8192])
def test_sign_verify_message_lengths(dil, oracle, mode, mlen):
    n = 9
    pk, sk = oracle.keypair_batch(mode, n, rand_index=5 + mlen)
    rng = np.random.default_rng(mlen)
    m = rng.integers(0, 256, (n, mlen), dtype=np.uint8)
    sig = dil[mode].sign(m, sk, exec_threshold=32)
    assert np.array_equal(sig, oracle.sign_batch(mode, m, sk))
    assert np.all(dil[mode].verify(sig, m, pk) == 0)


@pytest.mark.parametrize("mode", MODES)
def test_verify_rejects_tampering(dil, oracle, mode):
    p = oracle.params(mode)
    n = 64
    pk, sk = oracle.keypair_batch(mode, n, rand_index=31)
    m = messages(n, 64)
    sig = oracle.sign_batch(mode, m, sk)
    rng = np.random.default_rng(17)
    bad = sig.copy()
    flipped = rng.permutation(n)[: n // 2]
    for i in flipped:
        pos = int(rng.integers(0, p.sig_bytes))
        bad[i, pos] ^= np.uint8(1 << int(rng.integers(0, 8)))
    ret = dil[mode].verify(bad, m, pk)
    oret = oracle.verify_batch(mode, bad, m, pk)
    assert np.array_equal(ret, oret)
    # a flipped bit either breaks the signature or hits an unused hint byte that must be zero
    assert np.all(ret[flipped] == -1)
    untouched = np.setdiff1d(np.arange(n), flipped)
    assert np.all(ret[untouched] == 0)


@pytest.mark.parametrize("mode", MODES)
def test_verify_hint_encoding_checks(dil, oracle, mode):
    p = oracle.params(mode)
    h0 = 32 + p.l * p.polyz_packed
    pk, sk = oracle.keypair_batch(mode, 4, rand_index=77)
    m = messages(4, 32)
    sig = oracle.sign_batch(mode, m, sk)
    bad = sig.copy()
    bad[0, h0 + p.omega] = p.omega + 1             # count above omega
    bad[1, h0 + p.omega + p.k - 1] = 0             # counts decreasing
    bad[2, h0 + p.omega - 1] = 1                   # padding not zero (if unused)
    cnt0 = int(sig[3, h0 + p.omega])
    if cnt0 >= 2:
        bad[3, h0], bad[3, h0 + 1] = sig[3, h0 + 1], sig[3, h0]  # positions out of order
    ret = dil[mode].verify(bad, m, pk)
    assert np.array_equal(ret, oracle.verify_batch(mode, bad, m, pk))
    assert ret[0] == -1 and ret[1] == -1


@pytest.mark.parametrize("mode", MODES)
def test_verify_wrong_siglen_and_wrong_key(dil, oracle, mode):
    pk, sk = oracle.keypair_batch(mode, 6, rand_index=3)
    m = messages(6, 32)
    sig = oracle.sign_batch(mode, m, sk)
    p = oracle.params(mode)
    assert np.all(dil[mode].verify(sig, m, pk, siglen=p.sig_bytes + 1) == -1)
    ret = dil[mode].verify(sig, m, np.roll(pk, 1, axis=0))
    assert np.all(ret == -1)


def test_zero_batch_is_noop(dil):
    d = dil[2]
    pk, sk = d.keypair(0)
    assert pk.shape == (0, d.CRYPTO_PUBLICKEYBYTES)


def test_sign_lut_length_mismatch_is_an_error(dil, oracle):
    import torch
    from cudilithium_b200 import CudilError, TaskLut, alloc_pool, pinned
    d = dil[2]
    pk, sk = oracle.keypair_batch(2, 4)
    pool, sp = alloc_pool(d.sign_row_bytes(32), 4)
    tpool, tp = alloc_pool(d.sign_temp_row_bytes(), 8)
    lut = TaskLut(3, 8)  # the reference would spin forever here (src/api.cu:437-441)
    with pytest.raises(CudilError):
        d.crypto_sign_signature(pinned(4 * d.CRYPTO_BYTES), d.CRYPTO_BYTES, [0], pinned(128), 32, 32,
                                pinned(4 * d.CRYPTO_SECRETKEYBYTES), pool, sp, tpool, tp, lut, 8, 4)
    torch.cuda.synchronize()


def test_ntt_mul_matches_oracle(cuda_ok, oracle):
    import torch
    from cudilithium_b200 import ntt_mul
    q = 8380417
    rng = np.random.default_rng(42)
    n = 5000
    a = rng.integers(0, q, (n, 256), dtype=np.int64).astype(np.int32)
    b = rng.integers(0, q, (n, 256), dtype=np.int64).astype(np.int32)
    out = ntt_mul(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()).cpu().numpy()
    assert np.array_equal(out, oracle.ntt_mul_batch(a, b))
    # extreme inputs: all q-1, all 0, alternating
    a2 = np.stack([np.full(256, q - 1), np.zeros(256), np.tile([0, q - 1], 128)]).astype(np.int32)
    b2 = np.stack([np.full(256, q - 1), np.full(256, q - 1), np.full(256, -(q - 1))]).astype(np.int32)
    out2 = ntt_mul(torch.from_numpy(a2).cuda(), torch.from_numpy(b2).cuda()).cpu().numpy()
    assert np.array_equal(out2, oracle.ntt_mul_batch(a2, b2))
