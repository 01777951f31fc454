"""Request server (continuous batching, cudil_serve_trace), per-item message lengths of the plain
path and key-cache sharing between engines (needs a B200).

The serving tests check that every request's result is the same alone and in the mix: served in
mixed batches (fused and plain paths), served as a one-request trace, and computed by the CPU
oracle, signatures must be byte-identical and verify statuses equal the expected ones."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MODES = [2, 3, 5]


def oracle_keys(oracle, counts, base=4000):
    from cudilithium_b200.serve import Keys
    k = Keys()
    for m, n in counts.items():
        pk, sk = oracle.keypair_batch(m, n, rand_index=base + m)
        k.pk[m], k.sk[m] = pk.reshape(-1), sk.reshape(-1)
    return k


def request_msg(tr, i):
    o, l = int(tr.reqs["msg_off"][i]), int(tr.reqs["mlen"][i])
    return tr.msgs[o: o + l]


def oracle_sig(oracle, keys, tr, i):
    m = int(tr.reqs["mode"][i])
    p = oracle.params(m)
    k = int(tr.reqs["key"][i])
    sk = keys.sk[m].reshape(-1, p.sk_bytes)[k: k + 1]
    msg = request_msg(tr, i).reshape(1, -1)
    return oracle.sign_batch(m, msg, sk)[0]


def one_request_trace(tr, i):
    from cudilithium_b200.serve import Trace, VERIFY
    r = tr.reqs[i: i + 1].copy()
    r["arrival_s"] = 0.0
    msg = request_msg(tr, i)
    r["msg_off"] = 0
    sigs = np.zeros(8, np.uint8)
    if r["op"][0] == VERIFY:
        from cudilithium_b200 import _lib
        sb = _lib.params(int(r["mode"][0])).sig_bytes
        o = int(r["sig_off"][0])
        sigs = tr.sigs[o: o + sb].copy()
        r["sig_off"] = 0
    return Trace(r, np.concatenate([msg, np.zeros(8, np.uint8)]), sigs, tr.expect[i: i + 1], float("inf"))


@pytest.fixture(scope="module")
def mixed(oracle, cuda_ok):
    from cudilithium_b200.serve import poisson_trace
    keys = oracle_keys(oracle, {2: 40, 3: 24, 5: 24})
    tr = poisson_trace(keys, rate=40_000.0, n=900, seed=3, mlen_range=(0, 600), tamper_frac=0.15)
    return keys, tr


def check_results(tr, res, sigs, oracle, keys, sample):
    from cudilithium_b200 import _lib
    from cudilithium_b200.serve import SIGN
    assert np.all(res["done_s"] > 0)
    assert np.all(res["done_s"] >= tr.reqs["arrival_s"])
    ver = tr.reqs["op"] != SIGN
    assert np.array_equal(res["status"][ver], tr.expect[ver])
    for i in sample:
        if tr.reqs["op"][i] == SIGN:
            sb = _lib.params(int(tr.reqs["mode"][i])).sig_bytes
            assert np.array_equal(sigs[i, :sb], oracle_sig(oracle, keys, tr, i)), f"request {i}"


def expected_slots(tr, per_lane):
    """Slots of a load-weighted server: round(share * per_lane * lanes) per lane, at least per_lane."""
    from cudilithium_b200.serve import MODES
    lanes = [(m, op) for m in MODES for op in (0, 1) if ((tr.reqs["mode"] == m) & (tr.reqs["op"] == op)).any()]
    total = per_lane * len(lanes)
    n = len(tr.reqs)
    return sum(max(per_lane, int(total * ((tr.reqs["mode"] == m) & (tr.reqs["op"] == op)).sum() / n + 0.5))
               for m, op in lanes)


def test_serve_fused_mix_matches_oracle_and_alone(mixed, oracle):
    from cudilithium_b200 import _lib
    from cudilithium_b200.serve import SIGN, serve
    keys, tr = mixed
    assert tr.expect.min() == -1 and (tr.reqs["op"] == SIGN).sum() > 100
    res, sigs, st = serve(tr, keys, path=0, slots_per_lane=2, max_batch=64)
    assert st["slots"] == expected_slots(tr, 2) and st["batches"] >= 12
    assert res["batch_size"].max() > 1  # requests really shared batches
    sign_idx = np.nonzero(tr.reqs["op"] == SIGN)[0]
    check_results(tr, res, sigs, oracle, keys, sign_idx)
    # the same requests served alone
    rng = np.random.default_rng(5)
    for i in rng.choice(len(tr.reqs), 10, replace=False):
        tr1 = one_request_trace(tr, int(i))
        r1, s1, _ = serve(tr1, keys, path=0, slots_per_lane=1, max_batch=4)
        assert r1["status"][0] == res["status"][i] and r1["batch_size"][0] == 1
        if tr.reqs["op"][i] == SIGN:
            sb = _lib.params(int(tr.reqs["mode"][i])).sig_bytes
            assert np.array_equal(s1[0, :sb], sigs[i, :sb])


def test_serve_plain_equals_fused(mixed, oracle):
    from cudilithium_b200.serve import SIGN, serve
    keys, tr = mixed
    rf, sf, _ = serve(tr, keys, path=0, slots_per_lane=1, max_batch=128)
    rp, sp, st = serve(tr, keys, path=1, slots_per_lane=2, max_batch=96, plain_exec_threshold=256, slots_by_load=False)
    assert st["slots"] == 12
    assert np.array_equal(rp["status"], rf["status"])
    sign = tr.reqs["op"] == SIGN
    assert np.array_equal(sp[sign], sf[sign])
    check_results(tr, rp, sp, oracle, keys, np.nonzero(sign)[0][:40])


def test_serve_budget_admission(mixed, oracle):
    from cudilithium_b200._lib import CUDIL_ERR_BUDGET, CudilError
    from cudilithium_b200.serve import serve
    keys, tr = mixed
    with pytest.raises(CudilError) as ei:
        serve(tr, keys, path=1, budget_bytes=1 << 20, slots_per_lane=2, max_batch=64, plain_exec_threshold=128)
    assert ei.value.code == CUDIL_ERR_BUDGET
    # enough for one slot per lane but not two: admission keeps six slots and every result holds
    _, _, full = serve(tr, keys, path=1, slots_per_lane=1, max_batch=64, plain_exec_threshold=128, slots_by_load=False)
    res, sigs, st = serve(tr, keys, path=1, budget_bytes=int(full["device_bytes"] * 1.3), slots_per_lane=2,
                          max_batch=64, plain_exec_threshold=128, slots_by_load=False)
    assert 6 <= st["slots"] < 12 and st["device_bytes"] <= int(full["device_bytes"] * 1.3)
    check_results(tr, res, sigs, oracle, keys, np.nonzero(tr.reqs["op"] == 0)[0][:20])


def test_serve_invalid_trace(mixed):
    from cudilithium_b200._lib import CUDIL_ERR_INVALID, CudilError
    from cudilithium_b200.serve import Trace, serve
    keys, tr = mixed
    bad = tr.reqs.copy()
    bad["arrival_s"][5], bad["arrival_s"][6] = bad["arrival_s"][6], bad["arrival_s"][5] - 1.0  # out of order
    with pytest.raises(CudilError) as ei:
        serve(Trace(bad, tr.msgs, tr.sigs, tr.expect, tr.rate), keys, path=0)
    assert ei.value.code == CUDIL_ERR_INVALID
    bad = tr.reqs.copy()
    bad["key"][0] = 10_000  # no such key
    with pytest.raises(CudilError):
        serve(Trace(bad, tr.msgs, tr.sigs, tr.expect, tr.rate), keys, path=0)


@pytest.mark.parametrize("mode", MODES)
def test_plain_varlen_sign_verify(cuda_ok, oracle, mode):
    """cudil_sign_dev_varlen / cudil_verify_dev_varlen: per-item message lengths in one batch."""
    import ctypes

    import torch
    from cudilithium_b200 import _lib
    from cudilithium_b200._lib import check, lib
    from cudilithium_b200.api import TaskLut, alloc_pool
    rng = np.random.default_rng(90 + mode)
    p = oracle.params(mode)
    n, maxl = 130, 300
    pk, sk = oracle.keypair_batch(mode, n, rand_index=7000 + mode)
    lens = rng.integers(0, maxl + 1, n).astype(np.uint32)
    lens[:5] = [0, 1, 135, 136, maxl]
    m = rng.integers(0, 256, (n, maxl), dtype=np.uint8)
    want = oracle.sign_batch(mode, m, sk, mlens=lens)
    dev = torch.device("cuda")
    d_m = torch.from_numpy(m.reshape(-1)).to(dev)
    d_l = torch.from_numpy(lens.view(np.int32)).to(dev)
    d_sk = torch.from_numpy(sk.reshape(-1)).to(dev)
    d_sig = torch.zeros(n * p.sig_bytes, dtype=torch.uint8, device=dev)
    T = 64
    pool, sp = alloc_pool(lib.cudil_sign_row_bytes(mode, maxl), n)
    tpool, tp = alloc_pool(lib.cudil_sign_temp_row_bytes(mode), T)
    lut = TaskLut(n, T)
    check(lib.cudil_sign_dev_varlen(mode, d_sig.data_ptr(), p.sig_bytes, d_m.data_ptr(), maxl, d_l.data_ptr(), maxl,
                                    d_sk.data_ptr(), pool.data_ptr(), sp, tpool.data_ptr(), tp, ctypes.byref(lut.c), T, n, None),
          "cudil_sign_dev_varlen")
    torch.cuda.synchronize()
    sig = d_sig.cpu().numpy().reshape(n, p.sig_bytes)
    assert np.array_equal(sig, want)

    sig_t = sig.copy()
    bad = rng.permutation(n)[:13]
    for i in bad:
        sig_t[i, int(rng.integers(0, p.sig_bytes))] ^= np.uint8(1 << int(rng.integers(0, 8)))
    d_sig.copy_(torch.from_numpy(sig_t.reshape(-1)))
    d_pk = torch.from_numpy(pk.reshape(-1)).to(dev)
    d_ret = torch.full((n,), 7, dtype=torch.int32, device=dev)
    vpool, vp = alloc_pool(lib.cudil_verify_row_bytes(mode, maxl), n)
    check(lib.cudil_verify_dev_varlen(mode, d_ret.data_ptr(), d_sig.data_ptr(), p.sig_bytes, p.sig_bytes,
                                      d_m.data_ptr(), maxl, d_l.data_ptr(), maxl, d_pk.data_ptr(), vpool.data_ptr(),
                                      vp, n, None), "cudil_verify_dev_varlen")
    torch.cuda.synchronize()
    ret = d_ret.cpu().numpy()
    expect = oracle.verify_batch(mode, sig_t, m, pk, mlens=lens)
    assert np.array_equal(ret, expect)
    assert set(np.nonzero(ret)[0]) == set(bad)


def test_engine_attach_keys(cuda_ok, oracle):
    import torch
    from cudilithium_b200._lib import CudilError
    from cudilithium_b200.engine import Engine
    mode, nk, n = 3, 9, 60
    rng = np.random.default_rng(11)
    pk, sk = oracle.keypair_batch(mode, nk, rand_index=8100)
    owner = Engine(mode, max_keys=nk, max_items=0)
    owner.set_secret_keys(torch.from_numpy(sk.reshape(-1)).cuda())
    owner.set_public_keys(torch.from_numpy(pk.reshape(-1)).cuda())
    a = Engine(mode, max_keys=0, max_items=n)
    b = Engine(mode, max_keys=0, max_items=n)
    a.attach_keys(owner)
    b.attach_keys(owner)
    with pytest.raises(CudilError):
        a.set_secret_keys(torch.from_numpy(sk.reshape(-1)).cuda())
    msgs = [bytes(rng.integers(0, 256, int(l), dtype=np.uint8)) for l in rng.integers(0, 200, n)]
    key_idx = rng.integers(0, nk, n).astype(np.uint32)
    sa = a.sign_np(msgs, key_idx)
    sb = b.sign_np(msgs, key_idx)
    assert np.array_equal(sa, sb)
    for i in range(0, n, 7):
        want = oracle.sign_batch(mode, np.frombuffer(msgs[i], np.uint8).reshape(1, -1), sk[key_idx[i]: key_idx[i] + 1])
        assert np.array_equal(sa[i], want[0])
    assert np.all(b.verify_np(sa, msgs, key_idx) == 0)
    for e in (a, b, owner):
        e.close()
