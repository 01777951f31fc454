"""cudil_verify_noalloc: verification for callers that cannot allocate device memory.

Some callers may not call cudaMalloc where they verify (device memory reserved up front by a
budget, latency-critical threads, hosts that own all allocations).  cudil_verify_noalloc keeps
its scratch in a fixed array inside the library instead of a caller-allocated pool.  This test
calls it through the C ABI twice in a row, with different inputs each time (so the second call
runs over whatever the first left in the shared array), and requires results identical to
cudil_verify's on the same inputs (bit-exact, the tolerance of every test here).  It must pass
alone in a fresh process and after the rest of the suite, so it lives in a file collected last.
"""
import ctypes
import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch(oracle, mode, n, mlen, seed):
    p = oracle.params(mode)
    pk, sk = oracle.keypair_batch(mode, n, rand_index=seed)
    m = np.stack([np.frombuffer(hashlib.shake_128(bytes([seed, i % 256, i // 256])).digest(mlen), dtype=np.uint8)
                  for i in range(n)])
    sig = oracle.sign_batch(mode, m, sk)
    rng = np.random.default_rng(seed)
    bad = rng.permutation(n)[: n // 3]
    for i in bad:
        sig[i, int(rng.integers(0, p.sig_bytes))] ^= np.uint8(1 << int(rng.integers(0, 8)))
    return sig, m, pk


def _stage(torch, sig, m, pk):
    """Pinned host copies of a batch and a pinned result array (host memory only)."""
    from cudilithium_b200.api import pinned
    hs, hm, hp = pinned(sig.size), pinned(max(m.size, 1)), pinned(pk.size)
    hs.numpy()[: sig.size] = sig.reshape(-1)
    hm.numpy()[: m.size] = m.reshape(-1)
    hp.numpy()[: pk.size] = pk.reshape(-1)
    ret = torch.full((m.shape[0],), 7, dtype=torch.int32, pin_memory=True)
    return hs, hm, hp, ret


def _call(lib, torch, mode, staged, sig, m):
    hs, hm, hp, ret = staged
    n, mlen = m.shape
    rc = lib.cudil_verify_noalloc(mode, ret.data_ptr(), hs.data_ptr(), sig.shape[1], sig.shape[1], hm.data_ptr(),
                                  mlen, mlen, hp.data_ptr(), n, None)
    assert rc == 0
    torch.cuda.synchronize()
    return ret.numpy().copy()


@pytest.mark.parametrize("mode", [2, 3, 5])
def test_verify_noalloc_matches_verify_twice(cuda_ok, oracle, mode):
    import torch
    from cudilithium_b200 import Dilithium
    from cudilithium_b200._lib import CUDIL_ERR_BUDGET, lib

    d = Dilithium(mode)
    first = _batch(oracle, mode, 96, 32, seed=mode)
    second = _batch(oracle, mode, 61, 200, seed=mode + 40)
    for k, (sig, m, pk) in enumerate((first, second)):
        staged = _stage(torch, sig, m, pk)
        # the first call may load the library's module (and its fixed array) on this device; from
        # then on a call must not take any device memory
        free0 = torch.cuda.mem_get_info()[0]
        got = _call(lib, torch, mode, staged, sig, m)
        if k:
            assert torch.cuda.mem_get_info()[0] >= free0, "cudil_verify_noalloc took device memory"
        want = d.verify(sig, m, pk)
        assert np.array_equal(got, want)
        assert np.any(got == 0) and np.any(got == -1)

    cap = lib.cudil_verify_noalloc_max_batch(mode, 32)
    assert cap > 0
    rc = lib.cudil_verify_noalloc(mode, None, None, 0, d.CRYPTO_BYTES, None, 32, 32, None, cap + 1, None)
    assert rc == CUDIL_ERR_BUDGET
