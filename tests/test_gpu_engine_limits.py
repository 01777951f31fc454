"""Bounded device-side loops of the persistent signers (needs a B200).

Every loop of the signers that waits or retries has a run-time bound (cudil_engine_set_limits):
the per-item publication lock, the asynchronous signer's idle polls and the number of nonces an
item may try.  These tests make each bound run out on purpose -- with a limit of zero or one, so
that nothing waits long and nothing faults -- and check that the engine reports it through
cudil_engine_last_status, writes no signature it could not finish, and then signs the next batch
bit-exact with the oracle.  The reference has no such bound: its host loop waits for every item of
the task LUT (src/api.cu:437-441)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FILL = 0xA5


def _setup(oracle, mode, n, nk, seed):
    import torch

    from cudilithium_b200.engine import pack_messages
    rng = np.random.default_rng(seed)
    pk, sk = oracle.keypair_batch(mode, nk, rand_index=seed)
    m = rng.integers(0, 256, (n, 48), dtype=np.uint8)
    key_idx = (np.arange(n) % nk).astype(np.uint32)
    want, att = oracle.sign_batch(mode, m, sk[key_idx], return_attempts=True)
    d_msgs, offs, lens = pack_messages(m)
    d_sk = torch.from_numpy(sk.reshape(-1)).cuda()
    return d_sk, d_msgs, offs, lens, key_idx, want, att


def _sign_raw(eng, d_msgs, offs, lens, key_idx, n):
    """Signs into a buffer pre-filled with FILL; returns (rows, last_status rc, error bits)."""
    import torch

    from cudilithium_b200._lib import lib
    d_sig = torch.full((n * eng.params.sig_bytes,), FILL, dtype=torch.uint8, device="cuda")
    eng.sign(d_sig, d_msgs, offs, lens, key_idx)
    torch.cuda.synchronize()
    a, e = ctypes.c_ulonglong(), ctypes.c_uint32()
    rc = lib.cudil_engine_last_status(eng.h, ctypes.byref(a), ctypes.byref(e))
    return d_sig.cpu().numpy().reshape(n, -1), rc, e.value


@pytest.mark.parametrize("variant", [0, 1])
def test_lock_wait_runs_out_then_recovers(cuda_ok, oracle, variant):
    from cudilithium_b200._lib import CUDIL_ERR_TIMEOUT, CUDIL_OK
    from cudilithium_b200.engine import Engine
    mode, n = 2, 40
    d_sk, d_msgs, offs, lens, key_idx, want, _ = _setup(oracle, mode, n, 8, 61)
    eng = Engine(mode, max_keys=8, max_items=n)
    eng.set_sign_kernel(variant)
    eng.set_secret_keys(d_sk)
    # zero tries for the publication lock: every accepted attempt gives up before publishing
    eng.set_limits(lock_spins=0)
    rows, rc, err = _sign_raw(eng, d_msgs, offs, lens, key_idx, n)
    assert rc == CUDIL_ERR_TIMEOUT and (err & 1)
    assert np.all(rows == FILL)
    # the winners were still decided: the winning nonces are the deterministic ones
    eng.set_limits()
    rows, rc, err = _sign_raw(eng, d_msgs, offs, lens, key_idx, n)
    assert rc == CUDIL_OK and err == 0
    assert np.array_equal(rows, want)


def test_idle_limit_runs_out_then_recovers(cuda_ok, oracle):
    from cudilithium_b200._lib import CUDIL_ERR_TIMEOUT, CUDIL_OK
    from cudilithium_b200.engine import Engine
    mode, n = 3, 300
    d_sk, d_msgs, offs, lens, key_idx, want, _ = _setup(oracle, mode, n, 10, 62)
    eng = Engine(mode, max_keys=10, max_items=n)
    eng.set_sign_kernel(1)
    eng.set_secret_keys(d_sk)
    # no idle poll allowed: a warp that finds no ready job on its first look ends its block
    eng.set_limits(idle_polls=0)
    rows, rc, err = _sign_raw(eng, d_msgs, offs, lens, key_idx, n)
    assert rc == CUDIL_ERR_TIMEOUT and (err & 4)
    # whatever a block finished before it gave up is a correct signature; the rest is untouched
    done = ~np.all(rows == FILL, axis=1)
    assert np.array_equal(rows[done], want[done])
    eng.set_limits()
    rows, rc, err = _sign_raw(eng, d_msgs, offs, lens, key_idx, n)
    assert rc == CUDIL_OK and err == 0
    assert np.array_equal(rows, want)


@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("mode", [2, 5])
def test_nonce_limit_marks_exhausted_items(cuda_ok, oracle, mode, variant):
    from cudilithium_b200._lib import CUDIL_ERR_TIMEOUT, CUDIL_OK
    from cudilithium_b200.engine import Engine
    n = 64
    d_sk, d_msgs, offs, lens, key_idx, want, att = _setup(oracle, mode, n, 16, 63 + mode)
    assert (att == 1).any() and (att > 2).any()
    eng = Engine(mode, max_keys=16, max_items=n)
    eng.set_sign_kernel(variant)
    eng.set_secret_keys(d_sk)
    # two nonces per item: items the deterministic signer accepts at nonce 0 or 1 get their
    # signature, the others end as exhausted (their rows untouched) and the kernel still exits
    eng.set_limits(nonce_limit=2)
    rows, rc, err = _sign_raw(eng, d_msgs, offs, lens, key_idx, n)
    nonces = eng.last_nonces(n)
    ok = att <= 2
    assert rc == CUDIL_ERR_TIMEOUT and (err & 2)
    assert np.array_equal(nonces[ok] + 1, att[ok])
    assert np.all(nonces[~ok] == 0xFFFFFFFE)
    assert np.array_equal(rows[ok], want[ok])
    assert np.all(rows[~ok] == FILL)
    eng.set_limits()
    rows, rc, err = _sign_raw(eng, d_msgs, offs, lens, key_idx, n)
    assert rc == CUDIL_OK and err == 0
    assert np.array_equal(rows, want)
    # winning nonce + 1 = the deterministic signer's attempt count, item by item
    assert np.array_equal(eng.last_nonces(n) + 1, att)


def test_limits_argument_errors(cuda_ok):
    from cudilithium_b200 import CudilError
    from cudilithium_b200.engine import Engine
    eng = Engine(2, max_keys=1, max_items=4)
    with pytest.raises(CudilError):
        eng.set_limits(nonce_limit=0)
    with pytest.raises(CudilError):
        eng.set_limits(nonce_limit=65537)
    with pytest.raises(CudilError):
        eng.last_nonces(1)      # no signing batch yet
