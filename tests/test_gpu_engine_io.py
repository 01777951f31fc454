"""Fused engine input/output paths (needs a B200): key-cache rows built or replaced by key range,
and signatures written straight into pinned host memory by the signer, against the CPU oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _oracle_sign(oracle, mode, sk, key_idx, msgs):
    out = []
    for i, m in enumerate(msgs):
        arr = np.frombuffer(m, dtype=np.uint8).reshape(1, -1) if m else np.zeros((1, 0), np.uint8)
        out.append(oracle.sign_batch(mode, arr, sk[key_idx[i]: key_idx[i] + 1])[0])
    return np.stack(out)


@pytest.mark.parametrize("mode", [2, 3, 5])
@pytest.mark.parametrize("variant", [0, 3])
def test_chunked_key_build_and_host_output_match_oracle(cuda_ok, oracle, mode, variant):
    """Caches built in three key ranges; signatures into pinned host memory (4-byte aligned rows for
    Dilithium2, byte-aligned rows for Dilithium3/5), then into device memory, then into host memory
    again through a re-captured graph: every output equals the oracle."""
    import torch
    from cudilithium_b200 import Dilithium
    from cudilithium_b200.engine import Engine, pack_messages
    rng = np.random.default_rng(300 + 10 * mode + variant)
    nk, n = 9, 120
    p = Dilithium(mode).params
    pk, sk = oracle.keypair_batch(mode, nk, rand_index=4000 + mode)
    lens = rng.integers(0, 200, n)
    msgs = [bytes(rng.integers(0, 256, int(l), dtype=np.uint8)) for l in lens]
    key_idx = rng.integers(0, nk, n).astype(np.uint32)
    want = _oracle_sign(oracle, mode, sk, key_idx, msgs)
    eng = Engine(mode, max_keys=nk, max_items=n)
    eng.set_sign_kernel(variant)
    d_sk = torch.from_numpy(sk.reshape(-1)).cuda()
    for lo, hi in ((0, 4), (4, 5), (5, 9)):
        eng.update_secret_keys(d_sk[lo * p.sk_bytes: hi * p.sk_bytes], lo)
    d_msgs, offs, lens = pack_messages(msgs)
    h_sig = torch.zeros(n * p.sig_bytes, dtype=torch.uint8, pin_memory=True)
    eng.sign(h_sig, d_msgs, offs, lens, key_idx)
    torch.cuda.synchronize()
    assert np.array_equal(h_sig.numpy().reshape(n, -1), want)
    d_sig = torch.zeros(n * p.sig_bytes, dtype=torch.uint8, device="cuda")
    eng.sign(d_sig, d_msgs, offs, lens, key_idx)
    torch.cuda.synchronize()
    assert np.array_equal(d_sig.cpu().numpy().reshape(n, -1), want)
    h_sig.zero_()
    eng.sign(h_sig, d_msgs, offs, lens, key_idx)
    torch.cuda.synchronize()
    assert np.array_equal(h_sig.numpy().reshape(n, -1), want)
    assert eng.last_status()[1] == 0


def test_update_secret_keys_replaces_rows(cuda_ok, oracle):
    """Replacing rows 2..3 of a resident key table: items on those rows sign with the new keys,
    the other rows are untouched."""
    import torch
    from cudilithium_b200.engine import Engine
    mode, nk = 2, 6
    _, sk_a = oracle.keypair_batch(mode, nk, rand_index=10)
    _, sk_b = oracle.keypair_batch(mode, 2, rand_index=20)
    eng = Engine(mode, max_keys=nk, max_items=nk)
    eng.set_secret_keys(torch.from_numpy(sk_a.reshape(-1)).cuda())
    eng.update_secret_keys(torch.from_numpy(sk_b.reshape(-1)).cuda(), 2)
    table = sk_a.copy()
    table[2:4] = sk_b
    msgs = [b"row %d" % i for i in range(nk)]
    key_idx = np.arange(nk, dtype=np.uint32)
    assert np.array_equal(eng.sign_np(msgs, key_idx), _oracle_sign(oracle, mode, table, key_idx, msgs))


def test_update_secret_keys_and_output_errors(cuda_ok, oracle):
    """Ranges that would leave unbuilt rows inside the table or run past max_keys are refused, and
    so is pageable host memory as the signature output (before anything is queued)."""
    import torch
    from cudilithium_b200 import CudilError
    from cudilithium_b200.engine import Engine, pack_messages
    _, sk = oracle.keypair_batch(2, 3)
    d_sk = torch.from_numpy(sk.reshape(-1)).cuda()
    eng = Engine(2, max_keys=4, max_items=4)
    with pytest.raises(CudilError):
        eng.update_secret_keys(d_sk[: 2 * 2560], 1)   # row 0 not built yet
    eng.update_secret_keys(d_sk[: 2 * 2560], 0)
    with pytest.raises(CudilError):
        eng.update_secret_keys(d_sk, 2)               # rows 2..4 > max_keys
    eng.update_secret_keys(d_sk[: 2 * 2560], 2)       # rows 2..3: table full
    d_msgs, offs, lens = pack_messages([b"abc"] * 4)
    pageable = torch.zeros(4 * 2420, dtype=torch.uint8)
    with pytest.raises(CudilError):
        eng.sign(pageable, d_msgs, offs, lens, [0, 1, 2, 3])
    d_sig = torch.zeros(4 * 2420, dtype=torch.uint8, device="cuda")
    eng.sign(d_sig, d_msgs, offs, lens, [0, 1, 2, 3])
    torch.cuda.synchronize()
    table = np.concatenate([sk[:2], sk[:2]])
    want = _oracle_sign(oracle, 2, table, np.arange(4), [b"abc"] * 4)
    assert np.array_equal(d_sig.cpu().numpy().reshape(4, -1), want)
