"""The benchmark configurations at their full sizes, and the plain path at its maximum batch
(needs a B200).  The oracle is too slow to check every item at these sizes, so each test combines
size-independent properties (fused == plain over every item, every valid signature verifies,
exactly the tampered ones are rejected) with oracle checks on samples that include the extremes
(first and last items, the longest messages)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_ntt_microbench_full_size(cuda_ok, oracle):
    """2^20 polynomials, NTT -> Montgomery product -> invNTT: samples across the whole batch."""
    import torch

    from cudilithium_b200.api import ntt_mul
    npoly = 1 << 20
    g = torch.Generator(device="cuda").manual_seed(42)
    a = torch.randint(0, 8380417, (npoly, 256), dtype=torch.int32, device="cuda", generator=g)
    b = torch.randint(0, 8380417, (npoly, 256), dtype=torch.int32, device="cuda", generator=g)
    o = ntt_mul(a, b)
    torch.cuda.synchronize()
    rng = np.random.default_rng(1)
    idx = np.unique(np.concatenate([[0, 1, npoly - 2, npoly - 1], rng.integers(0, npoly, 2000)]))
    ti = torch.from_numpy(idx).cuda()
    want = oracle.ntt_mul_batch(a[ti].cpu().numpy(), b[ti].cpu().numpy())
    assert np.array_equal(o[ti].cpu().numpy(), want)


def _packed_messages(rng, lens):
    offs = np.zeros(len(lens), np.uint64)
    offs[1:] = np.cumsum((lens[:-1].astype(np.uint64) + 7) // 8 * 8)
    total = int(offs[-1] + lens[-1]) + 8
    return offs, rng.integers(0, 256, total, dtype=np.uint8)


def test_d3_loguniform_sign_full_size(cuda_ok, oracle):
    """Config 3: 16 384 Dilithium3 messages over 1024 keys, log-uniform 32 B .. 64 KiB."""
    import ctypes

    import torch

    import cudilithium_b200 as cd
    from cudilithium_b200 import _lib
    from cudilithium_b200.api import TaskLut, alloc_pool
    from cudilithium_b200.engine import Engine
    mode, nk, nm = 3, 1024, 16384
    d = cd.Dilithium(mode)
    p = d.params
    pk, sk = d.keypair(nk, rand_index=0)
    rng = np.random.default_rng(3)
    lens = np.floor(np.exp(rng.uniform(np.log(32), np.log(65536), nm))).astype(np.uint32)
    lens[123] = 65536
    offs, msgs = _packed_messages(rng, lens)
    keys = (np.arange(nm) % nk).astype(np.uint32)
    d_msgs = torch.from_numpy(msgs).cuda()
    eng = Engine(mode, nk, nm)
    eng.set_secret_keys(torch.from_numpy(sk.reshape(-1)).cuda())
    d_sig = torch.empty(nm * p.sig_bytes, dtype=torch.uint8, device="cuda")
    eng.sign(d_sig, d_msgs, offs, lens, keys)
    torch.cuda.synchronize()
    eng.last_status()
    # plain path over every item: pitched rows of the longest message
    mmax = int(lens.max())
    rows = np.zeros((nm, mmax), np.uint8)
    for i in range(nm):
        rows[i, : lens[i]] = msgs[int(offs[i]): int(offs[i]) + int(lens[i])]
    d_rows = torch.from_numpy(rows.reshape(-1)).cuda()
    del rows
    d_ml = torch.from_numpy(lens.astype(np.int32)).cuda()
    d_sk = torch.from_numpy(sk[keys].reshape(-1)).cuda()
    pool, sp = alloc_pool(d.sign_row_bytes(mmax), nm)
    tpool, tp = alloc_pool(d.sign_temp_row_bytes(), 8192)
    lut = TaskLut(nm, 8192)
    p_sig = torch.empty_like(d_sig)
    _lib.check(_lib.lib.cudil_sign_dev_varlen(mode, p_sig.data_ptr(), p.sig_bytes, d_rows.data_ptr(), mmax,
                                              d_ml.data_ptr(), mmax, d_sk.data_ptr(), pool.data_ptr(), sp,
                                              tpool.data_ptr(), tp, ctypes.byref(lut.c), 8192, nm, None), "sign")
    torch.cuda.synchronize()
    assert torch.equal(d_sig, p_sig)
    del pool, tpool, d_rows, d_sk
    ev = Engine(mode, nk, nm)
    ev.set_public_keys(torch.from_numpy(pk.reshape(-1)).cuda())
    d_ret = torch.empty(nm, dtype=torch.int32, device="cuda")
    ev.verify(d_ret, d_sig, d_msgs, offs, lens, keys)
    torch.cuda.synchronize()
    assert int((d_ret != 0).sum().item()) == 0
    sig = d_sig.cpu().numpy().reshape(nm, -1)
    sample = np.unique(np.concatenate([[0, nm - 1, 123], np.argsort(lens)[-4:], rng.integers(0, nm, 20)]))
    for i in sample:
        m = msgs[int(offs[i]): int(offs[i]) + int(lens[i])].reshape(1, -1)
        assert np.array_equal(sig[i], oracle.sign_batch(mode, m, sk[keys[i]: keys[i] + 1])[0]), i


def test_d5_cached_verify_full_size(cuda_ok, oracle):
    """Config 4: 65 536 Dilithium5 signatures (256 keys x 256 messages of 64 B), 10% bit-flipped."""
    import torch

    import cudilithium_b200 as cd
    from cudilithium_b200.engine import Engine
    mode, nk, nm = 5, 256, 65536
    d = cd.Dilithium(mode)
    p = d.params
    pk, sk = d.keypair(nk, rand_index=0)
    rng = np.random.default_rng(4)
    m = rng.integers(0, 256, (nm, 64), dtype=np.uint8)
    offs, lens = np.arange(nm, dtype=np.uint64) * 64, np.full(nm, 64, np.uint32)
    keys = (np.arange(nm) // 256).astype(np.uint32)
    d_m = torch.from_numpy(m.reshape(-1)).cuda()
    es = Engine(mode, nk, nm)
    es.set_secret_keys(torch.from_numpy(sk.reshape(-1)).cuda())
    d_sig = torch.empty(nm * p.sig_bytes, dtype=torch.uint8, device="cuda")
    es.sign(d_sig, d_m, offs, lens, keys)
    torch.cuda.synchronize()
    es.last_status()
    sig = d_sig.cpu().numpy().reshape(nm, -1)
    flip = rng.permutation(nm)[: nm // 10]
    for i in flip:
        sig[i, int(rng.integers(0, p.sig_bytes))] ^= np.uint8(1 << int(rng.integers(0, 8)))
    ev = Engine(mode, nk, nm)
    ev.set_public_keys(torch.from_numpy(pk.reshape(-1)).cuda())
    ret = ev.verify_np(sig, m, keys)
    expect = np.zeros(nm, np.int32)
    expect[flip] = -1
    assert np.array_equal(ret, expect)
    # the plain path (per-signature ExpandA and H(pk)) agrees on every signature
    assert np.array_equal(d.verify(sig, m, pk[keys]), expect)
    sample = np.unique(np.concatenate([[0, nm - 1], flip[:10], rng.integers(0, nm, 30)]))
    assert np.array_equal(oracle.verify_batch(mode, sig[sample], m[sample], pk[keys[sample]]), expect[sample])


def test_plain_path_maximum_batch(cuda_ok, oracle):
    """The plain path at the largest batch its exec slots can address (item << 16 | nonce: 65 536
    items), and one item more refused."""
    import ctypes

    import cudilithium_b200 as cd
    from cudilithium_b200._lib import CUDIL_ERR_INVALID, lib
    mode, n = 2, 65536
    d = cd.Dilithium(mode)
    pk, sk = d.keypair(n, rand_index=40000)
    m = oracle.messages_from_ctr(n, 32)
    sig = d.sign(m, sk, exec_threshold=16384)
    assert np.all(d.verify(sig, m, pk) == 0)
    rng = np.random.default_rng(5)
    sample = np.unique(np.concatenate([[0, 1, n - 2, n - 1], rng.integers(0, n, 30)]))
    assert np.array_equal(sig[sample], oracle.sign_batch(mode, m[sample], sk[sample]))
    siglen = ctypes.c_size_t(0)
    rc = lib.cudil_sign(mode, None, d.CRYPTO_BYTES, ctypes.byref(siglen), None, 32, 32, None, None, 0, None, 0,
                        None, 16384, n + 1, None)
    assert rc == CUDIL_ERR_INVALID
