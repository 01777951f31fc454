"""Signed-message format (sm = sig || m; cudil_crypto_sign / cudil_crypto_sign_open) against the
oracle and the detached-signature path (needs a B200)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MODES = [2, 3, 5]


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("mlen", [0, 1, 59])
def test_crypto_sign_and_open(cuda_ok, oracle, mode, mlen):
    import cudilithium_b200 as cd
    rng = np.random.default_rng(10 * mode + mlen)
    n = 33
    p = oracle.params(mode)
    pk, sk = oracle.keypair_batch(mode, n, rand_index=9900 + mode)
    m = rng.integers(0, 256, (n, mlen), dtype=np.uint8)
    d = cd.Dilithium(mode)
    sm = d.crypto_sign(m, sk)
    assert sm.shape == (n, p.sig_bytes + mlen)
    assert np.array_equal(sm[:, p.sig_bytes:], m)
    assert np.array_equal(sm[:, : p.sig_bytes], oracle.sign_batch(mode, m, sk))
    # open: valid rows give the message back, tampered rows give -1 and a zeroed message
    bad = sm.copy()
    flip = np.arange(0, n, 4)
    for i in flip:
        bad[i, int(rng.integers(0, bad.shape[1]))] ^= np.uint8(1 << int(rng.integers(0, 8)))
    got, ret, ml = d.crypto_sign_open(bad, pk)
    assert ml == mlen
    ok = np.ones(n, bool)
    ok[flip] = False
    assert np.all(ret[ok] == 0) and np.all(ret[~ok] == -1)
    assert np.array_equal(got[ok], m[ok]) and np.all(got[~ok] == 0)


def test_crypto_sign_open_short_input(cuda_ok, oracle):
    import cudilithium_b200 as cd
    pk, sk = oracle.keypair_batch(2, 3, rand_index=12)
    got, ret, ml = cd.Dilithium(2).crypto_sign_open(np.zeros((3, 100), np.uint8), pk)
    assert ml == 0 and np.all(ret == -1)
