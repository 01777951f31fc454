"""Randomized signing (rho' supplied by the caller instead of SHAKE256(K || mu); the reference's
DILITHIUM_RANDOMIZED_SIGNING, src/api.cu:143-148) on the plain path, the fused engine and the
api.cuh shim (needs a B200).  Given rho' the signature is deterministic, so it is checked bit for
bit against the oracle."""
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MODES = [2, 3, 5]


@pytest.mark.parametrize("mode", MODES)
def test_plain_randomized_matches_oracle(cuda_ok, oracle, mode):
    import cudilithium_b200 as cd
    rng = np.random.default_rng(500 + mode)
    n, mlen = 40, 77
    pk, sk = oracle.keypair_batch(mode, n, rand_index=5100 + mode)
    m = rng.integers(0, 256, (n, mlen), dtype=np.uint8)
    rp = rng.integers(0, 256, (n, 64), dtype=np.uint8)
    d = cd.Dilithium(mode)
    sig = d.sign(m, sk, exec_threshold=64, rhoprime=rp)
    for i in range(n):
        assert np.array_equal(sig[i], oracle.sign_rhoprime(mode, m[i].tobytes(), sk[i], rp[i].tobytes())), i
    assert np.all(d.verify(sig, m, pk) == 0)
    det = d.sign(m, sk, exec_threshold=64)
    assert not np.array_equal(det, sig)
    assert np.array_equal(det, oracle.sign_batch(mode, m, sk))


@pytest.mark.parametrize("mode", MODES)
def test_engine_randomized_matches_oracle(cuda_ok, oracle, mode):
    import torch
    from cudilithium_b200.engine import Engine
    rng = np.random.default_rng(600 + mode)
    nk, n = 4, 90
    pk, sk = oracle.keypair_batch(mode, nk, rand_index=6100 + mode)
    eng = Engine(mode, max_keys=nk, max_items=n)
    eng.set_secret_keys(torch.from_numpy(sk.reshape(-1)).cuda())
    eng.set_public_keys(torch.from_numpy(pk.reshape(-1)).cuda())
    msgs = [bytes(rng.integers(0, 256, int(l), dtype=np.uint8)) for l in rng.integers(0, 300, n)]
    key_idx = rng.integers(0, nk, n).astype(np.uint32)
    rp = rng.integers(0, 256, (n, 64), dtype=np.uint8)
    sig = eng.sign_np(msgs, key_idx, rhoprime=rp)
    for i in range(0, n, 3):
        want = oracle.sign_rhoprime(mode, msgs[i], sk[key_idx[i]], rp[i].tobytes())
        assert np.array_equal(sig[i], want), i
    assert np.all(eng.verify_np(sig, msgs, key_idx) == 0)
    # the deterministic graph is separate: it still gives the deterministic signatures
    det = eng.sign_np(msgs[:10], key_idx[:10])
    for i in range(10):
        m1 = np.frombuffer(msgs[i], np.uint8).reshape(1, -1) if msgs[i] else np.zeros((1, 0), np.uint8)
        assert np.array_equal(det[i], oracle.sign_batch(mode, m1, sk[key_idx[i]: key_idx[i] + 1])[0])


def test_api_shim_randomized_signatures_verify(tmp_path, cuda_ok, oracle):
    from test_api_shim import build_shim
    mode, n, mlen = 2, 64, 32
    exe = build_shim(mode, tmp_path, extra=["-DDILITHIUM_RANDOMIZED_SIGNING"])
    m = oracle.messages_from_ctr(n, mlen)
    (tmp_path / "m.bin").write_bytes(m.tobytes())
    r = subprocess.run([str(exe), str(tmp_path), str(n), str(mlen)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout
    p = oracle.params(mode)
    pk = np.fromfile(tmp_path / "pk.bin", np.uint8).reshape(n, p.pk_bytes)
    sig = np.fromfile(tmp_path / "sig.bin", np.uint8).reshape(n, p.sig_bytes)
    ret = np.fromfile(tmp_path / "ret.bin", np.int32)
    assert np.all(ret == 0)
    assert np.all(oracle.verify_batch(mode, sig, m, pk) == 0)
    sk = np.fromfile(tmp_path / "sk.bin", np.uint8).reshape(n, p.sk_bytes)
    det = oracle.sign_batch(mode, m, sk)
    assert sum(np.array_equal(sig[i], det[i]) for i in range(n)) == 0  # fresh rho' per message


def test_derive_rhoprime_matches_oracle(cuda_ok, oracle):
    """Device-side rho' derivation (cudil_derive_rhoprime) vs the oracle's restatement."""
    import torch

    from cudilithium_b200._lib import lib
    from cudilithium_b200.api import derive_rhoprime
    seed = bytes(range(100, 132))
    for counter, n in ((0, 1), (12345, 1000), (2**64 - 5, 10)):
        got = derive_rhoprime(seed, counter, n).cpu().numpy()
        assert np.array_equal(got, oracle.derive_rhoprime(seed, counter, n))
    # pitched, unaligned rows
    pitch, n = 77, 33
    buf = torch.zeros(n * pitch + 3, dtype=torch.uint8, device="cuda")
    assert lib.cudil_derive_rhoprime(buf.data_ptr() + 3, pitch, seed, 9, n, None) == 0
    torch.cuda.synchronize()
    rows = buf.cpu().numpy()[3:3 + n * pitch].reshape(n, pitch)[:, :64]
    assert np.array_equal(rows, oracle.derive_rhoprime(seed, 9, n))
    assert lib.cudil_derive_rhoprime(buf.data_ptr(), 63, seed, 0, 1, None) != 0


@pytest.mark.parametrize("mode", MODES)
def test_engine_seeded_matches_oracle(cuda_ok, oracle, mode):
    """Seeded randomized signing: rho' derived on the device inside the engine's prehash kernel."""
    import torch
    from cudilithium_b200.engine import Engine, pack_messages
    rng = np.random.default_rng(700 + mode)
    nk, n = 5, 70
    pk, sk = oracle.keypair_batch(mode, nk, rand_index=7100 + mode)
    eng = Engine(mode, max_keys=nk, max_items=n)
    eng.set_secret_keys(torch.from_numpy(sk.reshape(-1)).cuda())
    eng.set_public_keys(torch.from_numpy(pk.reshape(-1)).cuda())
    msgs = [bytes(rng.integers(0, 256, int(l), dtype=np.uint8)) for l in rng.integers(0, 400, n)]
    key_idx = rng.integers(0, nk, n).astype(np.uint32)
    seed = bytes(rng.integers(0, 256, 32, dtype=np.uint8))
    d_msgs, offs, lens = pack_messages(msgs)
    d_sig = torch.empty(n * eng.params.sig_bytes, dtype=torch.uint8, device="cuda")
    for counter, cnt in ((0, n), (2**40 + 7, 23)):          # two batches through the same graph
        eng.sign(d_sig, d_msgs, offs[:cnt], lens[:cnt], key_idx[:cnt], rho_seed=seed, rho_counter=counter)
        torch.cuda.synchronize()
        eng.last_status()
        sig = d_sig.cpu().numpy()[: cnt * eng.params.sig_bytes].reshape(cnt, -1)
        rps = oracle.derive_rhoprime(seed, counter, cnt)
        for i in range(0, cnt, 4):
            want = oracle.sign_rhoprime(mode, msgs[i], sk[key_idx[i]], rps[i].tobytes())
            assert np.array_equal(sig[i], want), (counter, i)
        assert np.all(eng.verify_np(sig, msgs[:cnt], key_idx[:cnt]) == 0)
    # a deterministic batch afterwards is unaffected by the previous batch's seed
    det = eng.sign_np(msgs[:8], key_idx[:8])
    for i in range(8):
        m1 = np.frombuffer(msgs[i], np.uint8).reshape(1, -1) if msgs[i] else np.zeros((1, 0), np.uint8)
        assert np.array_equal(det[i], oracle.sign_batch(mode, m1, sk[key_idx[i]: key_idx[i] + 1])[0])


def test_plain_with_device_derived_rhoprime(cuda_ok, oracle):
    """The plain path signing with rho' rows that the device derived from one seed."""
    import cudilithium_b200 as cd
    from cudilithium_b200.api import derive_rhoprime
    mode, n = 3, 24
    rng = np.random.default_rng(88)
    pk, sk = oracle.keypair_batch(mode, n, rand_index=88)
    m = rng.integers(0, 256, (n, 50), dtype=np.uint8)
    seed = bytes(rng.integers(0, 256, 32, dtype=np.uint8))
    rp = derive_rhoprime(seed, 5, n).cpu().numpy()
    sig = cd.Dilithium(mode).sign(m, sk, exec_threshold=32, rhoprime=rp)
    orp = oracle.derive_rhoprime(seed, 5, n)
    for i in range(n):
        assert np.array_equal(sig[i], oracle.sign_rhoprime(mode, m[i].tobytes(), sk[i], orp[i].tobytes())), i
