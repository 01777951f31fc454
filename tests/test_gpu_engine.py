"""Fused engine (persistent kernel + per-key caches + graph) vs the CPU oracle (needs a B200)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MODES = [2, 3, 5]


def rand_msgs(rng, n, lens):
    return [bytes(rng.integers(0, 256, int(l), dtype=np.uint8)) for l in lens]


def oracle_sign(oracle, mode, sk, key_idx, msgs):
    out = []
    for i, m in enumerate(msgs):
        arr = np.frombuffer(m, dtype=np.uint8).reshape(1, -1) if m else np.zeros((1, 0), np.uint8)
        out.append(oracle.sign_batch(mode, arr, sk[key_idx[i]: key_idx[i] + 1])[0])
    return np.stack(out)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("threads", [128, 256])
def test_engine_sign_matches_oracle(cuda_ok, oracle, mode, threads):
    import torch
    from cudilithium_b200.engine import Engine
    rng = np.random.default_rng(mode * 10 + threads)
    nk, n = 7, 150
    pk, sk = oracle.keypair_batch(mode, nk, rand_index=500 + mode)
    lens = rng.integers(0, 300, n)
    lens[:6] = [0, 1, 135, 136, 137, 8]
    msgs = rand_msgs(rng, n, lens)
    key_idx = rng.integers(0, nk, n).astype(np.uint32)
    eng = Engine(mode, max_keys=nk, max_items=n, threads=threads)
    eng.set_secret_keys(torch.from_numpy(sk.reshape(-1)).cuda())
    sig = eng.sign_np(msgs, key_idx)
    want = oracle_sign(oracle, mode, sk, key_idx, msgs)
    assert np.array_equal(sig, want)
    # second, smaller batch through the same graph (batch size lives in device memory)
    sig2 = eng.sign_np(msgs[:17], key_idx[:17])
    assert np.array_equal(sig2, want[:17])
    attempts, err = eng.last_status()
    assert err == 0 and attempts >= 17


@pytest.mark.parametrize("mode", MODES)
def test_engine_verify_matches_oracle(cuda_ok, oracle, mode):
    import torch
    from cudilithium_b200.engine import Engine
    rng = np.random.default_rng(70 + mode)
    nk, n = 5, 200
    p = oracle.params(mode)
    pk, sk = oracle.keypair_batch(mode, nk, rand_index=900 + mode)
    lens = rng.integers(0, 200, n)
    msgs = rand_msgs(rng, n, lens)
    key_idx = rng.integers(0, nk, n).astype(np.uint32)
    sig = oracle_sign(oracle, mode, sk, key_idx, msgs)
    flip = rng.permutation(n)[: n // 10]
    for i in flip:
        sig[i, int(rng.integers(0, p.sig_bytes))] ^= np.uint8(1 << int(rng.integers(0, 8)))
    eng = Engine(mode, max_keys=nk, max_items=n)
    eng.set_public_keys(torch.from_numpy(pk.reshape(-1)).cuda())
    ret = eng.verify_np(sig, msgs, key_idx)
    want = np.array([oracle.verify_batch(mode, sig[i:i + 1],
                                         np.frombuffer(msgs[i], np.uint8).reshape(1, -1) if msgs[i] else np.zeros((1, 0), np.uint8),
                                         pk[key_idx[i]: key_idx[i] + 1])[0] for i in range(n)])
    assert np.array_equal(ret, want)
    assert np.all(ret[flip] == -1)


def test_engine_matches_plain_path_large_batch(cuda_ok, oracle):
    """Dilithium2, 4000 messages over 300 keys: fused engine == plain stage-by-stage path."""
    import torch
    from cudilithium_b200 import Dilithium
    from cudilithium_b200.engine import Engine
    mode, nk, n = 2, 300, 4000
    d = Dilithium(mode)
    pk, sk = d.keypair(nk, rand_index=77)
    rng = np.random.default_rng(5)
    key_idx = rng.integers(0, nk, n).astype(np.uint32)
    m = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    plain = d.sign(m, sk[key_idx], exec_threshold=4096)
    eng = Engine(mode, max_keys=nk, max_items=n)
    eng.set_secret_keys(torch.from_numpy(sk.reshape(-1)).cuda())
    fused = eng.sign_np(m, key_idx)
    assert np.array_equal(fused, plain)
    veng = Engine(mode, max_keys=nk, max_items=n)
    veng.set_public_keys(torch.from_numpy(pk.reshape(-1)).cuda())
    assert np.all(veng.verify_np(fused, m, key_idx) == 0)


def test_engine_long_messages(cuda_ok, oracle):
    """Dilithium3 with message lengths up to 64 KiB (log-uniform), as the long-message workload."""
    import torch
    from cudilithium_b200.engine import Engine
    mode, nk, n = 3, 4, 24
    pk, sk = oracle.keypair_batch(mode, nk, rand_index=31)
    rng = np.random.default_rng(9)
    lens = np.floor(np.exp(rng.uniform(np.log(32), np.log(65536), n))).astype(int)
    lens[0] = 65536
    msgs = rand_msgs(rng, n, lens)
    key_idx = (np.arange(n) % nk).astype(np.uint32)
    eng = Engine(mode, max_keys=nk, max_items=n)
    eng.set_secret_keys(torch.from_numpy(sk.reshape(-1)).cuda())
    assert np.array_equal(eng.sign_np(msgs, key_idx), oracle_sign(oracle, mode, sk, key_idx, msgs))


def test_engine_argument_errors(cuda_ok, oracle):
    import torch
    from cudilithium_b200 import CudilError
    from cudilithium_b200._lib import CUDIL_ERR_BUDGET
    from cudilithium_b200.engine import Engine, pack_messages
    pk, sk = oracle.keypair_batch(2, 2)
    eng = Engine(2, max_keys=2, max_items=8)
    eng.set_secret_keys(torch.from_numpy(sk.reshape(-1)).cuda())
    d_msgs, offs, lens = pack_messages([b"abc"] * 4)
    d_sig = torch.empty(4 * 2420, dtype=torch.uint8, device="cuda")
    with pytest.raises(CudilError):
        eng.sign(d_sig, d_msgs, offs, lens, [0, 1, 2, 0])      # key index out of range
    with pytest.raises(CudilError):
        eng.sign(d_sig, d_msgs, offs + 1, lens, [0, 0, 0, 0])  # misaligned message offsets
    with pytest.raises(CudilError):
        eng.sign(d_sig, d_msgs, np.zeros(9, np.uint64), np.zeros(9, np.uint32), np.zeros(9, np.uint32))  # > max_items
    with pytest.raises(CudilError) as ei:
        Engine(5, max_keys=4096, max_items=65536, budget_bytes=1 << 20)
    assert ei.value.code == CUDIL_ERR_BUDGET


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5])
def test_engine_sign_kernel_variants_match_oracle(cuda_ok, oracle, mode, variant):
    """Every signer kernel (phased, the four asynchronous shapes, phased with one wide block per SM)
    gives the oracle's signatures: many items per block, fewer items than blocks, one item,
    repeated keys, uneven message lengths, and a batch where several blocks own no item."""
    import torch
    from cudilithium_b200.engine import Engine
    rng = np.random.default_rng(300 + 10 * mode + variant)
    nk = 5
    pk, sk = oracle.keypair_batch(mode, nk, rand_index=1300 + mode)
    eng = Engine(mode, max_keys=nk, max_items=700)
    eng.set_sign_kernel(variant)
    assert eng.info()["sign_blocks"] > 0
    eng.set_secret_keys(torch.from_numpy(sk.reshape(-1)).cuda())
    for n in (700, 97, 1):
        lens = rng.integers(0, 400, n)
        msgs = rand_msgs(rng, n, lens)
        key_idx = rng.integers(0, nk, n).astype(np.uint32)
        sig = eng.sign_np(msgs, key_idx)
        want = oracle_sign(oracle, mode, sk, key_idx, msgs)
        assert np.array_equal(sig, want), f"n={n}"
        attempts, err = eng.last_status()
        assert err == 0 and attempts >= n
    # the accepted signatures verify through the cached public keys
    eng.set_public_keys(torch.from_numpy(pk.reshape(-1)).cuda())
    assert np.all(eng.verify_np(sig, msgs, key_idx) == 0)


@pytest.mark.parametrize("large", [(100, 5, 128), (100, 2, 0), (0, 5, 0)])
def test_engine_large_batch_class(cuda_ok, oracle, large):
    """Batches at or above the large-batch threshold sign through the large-batch kernel and graph,
    smaller ones through the default: sizes alternate between the classes on one engine, and every
    result equals the oracle."""
    import torch
    from cudilithium_b200.engine import Engine
    mode, nk = 2, 4
    rng = np.random.default_rng(900 + large[1])
    pk, sk = oracle.keypair_batch(mode, nk, rand_index=3100)
    eng = Engine(mode, max_keys=nk, max_items=300)
    eng.set_large_batch(*large)
    eng.set_secret_keys(torch.from_numpy(sk.reshape(-1)).cuda())
    for n in (300, 40, 100, 99, 250):
        msgs = rand_msgs(rng, n, rng.integers(0, 200, n))
        key_idx = rng.integers(0, nk, n).astype(np.uint32)
        assert np.array_equal(eng.sign_np(msgs, key_idx), oracle_sign(oracle, mode, sk, key_idx, msgs)), f"n={n}"
        assert eng.last_status()[1] == 0


@pytest.mark.parametrize("variant", [1, 3, 5])
@pytest.mark.parametrize("spec", [1, 8, 0])
def test_engine_async_speculation_targets(cuda_ok, oracle, variant, spec):
    """Speculation target 1 (no speculation), 8 and the largest one give the same signatures."""
    import torch
    from cudilithium_b200.engine import Engine
    mode, nk, n = 2, 3, 400
    rng = np.random.default_rng(77 + spec + variant)
    pk, sk = oracle.keypair_batch(mode, nk, rand_index=2100)
    eng = Engine(mode, max_keys=nk, max_items=n)
    eng.set_sign_kernel(variant)
    eng.set_spec_slots(spec if spec else 1024)
    eng.set_secret_keys(torch.from_numpy(sk.reshape(-1)).cuda())
    msgs = rand_msgs(rng, n, rng.integers(0, 100, n))
    key_idx = rng.integers(0, nk, n).astype(np.uint32)
    assert np.array_equal(eng.sign_np(msgs, key_idx), oracle_sign(oracle, mode, sk, key_idx, msgs))


@pytest.mark.parametrize("mode", MODES)
def test_engine_single_item_capacity(cuda_ok, oracle, mode):
    """An engine sized for one item (smallest staging buffers) signs and verifies correctly."""
    import torch
    from cudilithium_b200.engine import Engine
    pk, sk = oracle.keypair_batch(mode, 2, rand_index=3100 + mode)
    eng = Engine(mode, max_keys=2, max_items=1)
    eng.set_secret_keys(torch.from_numpy(sk.reshape(-1)).cuda())
    eng.set_public_keys(torch.from_numpy(pk.reshape(-1)).cuda())
    msg = [b"single item capacity"]
    sig = eng.sign_np(msg, np.array([1], np.uint32))
    assert np.array_equal(sig, oracle_sign(oracle, mode, sk, [1], msg))
    assert eng.verify_np(sig, msg, np.array([1], np.uint32))[0] == 0
    assert eng.verify_np(sig, msg, np.array([0], np.uint32))[0] == -1


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("variant", [0, 3])
def test_engine_long_messages_match_oracle(cuda_ok, oracle, mode, variant):
    """Messages across SHAKE256 block boundaries up to 64 KiB (the log-uniform workload's range)
    sign and verify bit-exactly through the engine."""
    import torch
    from cudilithium_b200.engine import Engine
    rng = np.random.default_rng(40 + mode + variant)
    lens = [0, 1, 103, 104, 105, 135, 136, 137, 239, 240, 4095, 4096, 65536, 65535]
    n, nk = len(lens), 3
    pk, sk = oracle.keypair_batch(mode, nk, rand_index=4200 + mode)
    msgs = rand_msgs(rng, n, lens)
    key_idx = (np.arange(n) % nk).astype(np.uint32)
    eng = Engine(mode, max_keys=nk, max_items=n)
    eng.set_sign_kernel(variant)
    eng.set_secret_keys(torch.from_numpy(sk.reshape(-1)).cuda())
    eng.set_public_keys(torch.from_numpy(pk.reshape(-1)).cuda())
    sig = eng.sign_np(msgs, key_idx)
    assert np.array_equal(sig, oracle_sign(oracle, mode, sk, key_idx, msgs))
    assert np.all(eng.verify_np(sig, msgs, key_idx) == 0)
    bad = [m[:-1] + bytes([m[-1] ^ 1]) if m else b"x" for m in msgs]
    assert np.all(eng.verify_np(sig, bad, key_idx) == -1)


@pytest.mark.parametrize("mode", MODES)
def test_sign_pipeline_batches_match_oracle(cuda_ok, oracle, mode):
    """EnginePipeline: five batches of different messages over two engines on two streams (each
    batch rebuilds its engine's key caches), every batch's signatures equal the oracle's, and the
    same batches verify through the pipeline (a tampered signature is rejected)."""
    import torch
    from cudilithium_b200.engine import EnginePipeline, pack_messages
    rng = np.random.default_rng(400 + mode)
    nk, n, nb = 6, 40, 5
    p = oracle.params(mode)
    pk, sk = oracle.keypair_batch(mode, nk, rand_index=610 + mode)
    d_sk = torch.from_numpy(sk.reshape(-1)).cuda()
    pipe = EnginePipeline(mode, max_keys=nk, max_items=n, depth=2)
    batches, outs = [], []
    try:
        for b in range(nb):
            lens = rng.integers(0, 200, n)
            msgs = rand_msgs(rng, n, lens)
            key_idx = rng.integers(0, nk, n).astype(np.uint32)
            d_msgs, offs, mlens = pack_messages(msgs)
            d_sig = torch.empty(n * p.sig_bytes, dtype=torch.uint8, device="cuda")
            pipe.sign(d_sig, d_msgs, offs, mlens, key_idx, d_sk=d_sk, after=torch.cuda.current_stream())
            batches.append((msgs, key_idx, d_msgs, offs, mlens))
            outs.append(d_sig)
        pipe.join()
        torch.cuda.synchronize()
        for (msgs, key_idx, _, _, _), d_sig in zip(batches, outs):
            got = d_sig.cpu().numpy().reshape(n, p.sig_bytes)
            assert np.array_equal(got, oracle_sign(oracle, mode, sk, key_idx, msgs))
        for e in pipe.engines:
            assert e.last_status()[1] == 0
        # the same batches verified through the pipeline (public-key caches built per batch), one
        # signature of the last batch tampered with
        d_pk = torch.from_numpy(pk.reshape(-1)).cuda()
        outs[-1][p.sig_bytes * 3 + 50] ^= 1
        rets = []
        for (msgs, key_idx, d_msgs, offs, mlens), d_sig in zip(batches, outs):
            d_ret = torch.empty(n, dtype=torch.int32, device="cuda")
            pipe.verify(d_ret, d_sig, d_msgs, offs, mlens, key_idx, d_pk=d_pk, after=torch.cuda.current_stream())
            rets.append(d_ret)
        pipe.join()
        torch.cuda.synchronize()
        for b, d_ret in enumerate(rets):
            want = np.zeros(n, np.int32)
            if b == nb - 1:
                want[3] = -1
            assert np.array_equal(d_ret.cpu().numpy(), want)
    finally:
        pipe.close()


def test_pipeline_shared_keys_match_oracle(cuda_ok, oracle):
    """EnginePipeline(share_keys=True): the key caches are built once through the first engine and
    read by the second; four batches over the two engines equal the oracle's signatures."""
    import torch
    from cudilithium_b200.engine import EnginePipeline, pack_messages
    mode, nk, n = 3, 5, 30
    p = oracle.params(mode)
    rng = np.random.default_rng(77)
    pk, sk = oracle.keypair_batch(mode, nk, rand_index=720)
    pipe = EnginePipeline(mode, max_keys=nk, max_items=n, depth=2, share_keys=True)
    try:
        pipe.engines[0].set_secret_keys(torch.from_numpy(sk.reshape(-1)).cuda())
        batches = []
        for _ in range(4):
            msgs = rand_msgs(rng, n, rng.integers(0, 500, n))
            key_idx = rng.integers(0, nk, n).astype(np.uint32)
            d_msgs, offs, lens = pack_messages(msgs)
            d_sig = torch.empty(n * p.sig_bytes, dtype=torch.uint8, device="cuda")
            pipe.sign(d_sig, d_msgs, offs, lens, key_idx, after=torch.cuda.current_stream())
            batches.append((msgs, key_idx, d_msgs, d_sig))
        pipe.join()
        torch.cuda.synchronize()
        for msgs, key_idx, _, d_sig in batches:
            got = d_sig.cpu().numpy().reshape(n, p.sig_bytes)
            assert np.array_equal(got, oracle_sign(oracle, mode, sk, key_idx, msgs))
        # per-batch keys need caches of each engine's own: refused before anything is queued
        k0 = pipe.k
        msgs, key_idx, d_msgs, d_sig = batches[0]
        _, offs, lens = pack_messages(msgs)
        with pytest.raises(ValueError):
            pipe.sign(d_sig, d_msgs, offs, lens, key_idx, d_sk=torch.from_numpy(sk.reshape(-1)).cuda())
        assert pipe.k == k0
    finally:
        pipe.close()


@pytest.mark.parametrize("mode", MODES)
def test_public_key_cache_built_beside_signing(cuda_ok, oracle, mode):
    """The verifier's public-key cache is built on a second stream while another engine signs (the
    keygen + sign + verify sequence); verification on the first stream waits for both.  Signatures
    equal the oracle's, every one verifies, and a tampered one is rejected."""
    import torch
    from cudilithium_b200.engine import Engine, pack_messages
    rng = np.random.default_rng(140 + mode)
    nk, n = 6, 64
    p = oracle.params(mode)
    pk, sk = oracle.keypair_batch(mode, nk, rand_index=1300 + mode)
    msgs = rand_msgs(rng, n, rng.integers(0, 300, n))
    key_idx = rng.integers(0, nk, n).astype(np.uint32)
    d_msgs, offs, lens = pack_messages(msgs)
    es, ev = Engine(mode, max_keys=nk, max_items=n), Engine(mode, max_keys=nk, max_items=n)
    try:
        st = torch.cuda.current_stream()
        side = torch.cuda.Stream()
        d_pk = torch.from_numpy(pk.reshape(-1)).cuda()
        d_sk = torch.from_numpy(sk.reshape(-1)).cuda()
        keys_ready, pk_ready = torch.cuda.Event(), torch.cuda.Event()
        keys_ready.record(st)
        side.wait_event(keys_ready)
        ev.set_public_keys(d_pk, stream=side)
        pk_ready.record(side)
        d_sig = torch.empty(n * p.sig_bytes, dtype=torch.uint8, device="cuda")
        es.set_secret_keys(d_sk, stream=st)
        es.sign(d_sig, d_msgs, offs, lens, key_idx, stream=st)
        st.wait_event(pk_ready)
        d_sig[p.sig_bytes * 7] ^= 1  # item 7 tampered after signing, before verification
        ret = torch.full((n,), 7, dtype=torch.int32, device="cuda")
        ev.verify(ret, d_sig, d_msgs, offs, lens, key_idx, stream=st)
        torch.cuda.synchronize()
        want = oracle_sign(oracle, mode, sk, key_idx, msgs)
        want[7, 0] ^= 1
        assert np.array_equal(d_sig.cpu().numpy().reshape(n, p.sig_bytes), want)
        r = ret.cpu().numpy()
        assert r[7] == -1
        assert np.all(np.delete(r, 7) == 0)
    finally:
        es.close()
        ev.close()
