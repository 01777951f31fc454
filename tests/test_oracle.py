"""The CPU oracle against the reference's pinned golden values (no GPU)."""
import hashlib
import os
import random

import numpy as np
import pytest

MODES = [2, 3, 5]


@pytest.mark.parametrize("mode", MODES)
def test_oracle_reproduces_reference_tvecs_digest(oracle, golden_digests, mode):
    """sha256 of the regenerated tvecs file equals the reference's CTest digest."""
    data = oracle.tvecs(mode, golden_digests["nvectors"])
    assert hashlib.sha256(data).hexdigest() == golden_digests["sha256"][str(mode)]


def test_keccak_matches_hashlib(oracle):
    rng = random.Random(7)
    for n in [0, 1, 7, 33, 135, 136, 137, 167, 168, 169, 271, 272, 1000]:
        data = bytes(rng.getrandbits(8) for _ in range(n))
        for outlen in [1, 32, 136, 168, 500]:
            assert oracle.shake128(data, outlen) == hashlib.shake_128(data).digest(outlen)
            assert oracle.shake256(data, outlen) == hashlib.shake_256(data).digest(outlen)


def test_keccak_matches_reference_fips202(oracle):
    """Byte-for-byte against the reference's own src/fips202/fips202.c compiled into oracle/_ref."""
    import ctypes
    if not oracle.REF_LIB.exists():
        root = oracle.ref_root()
        if root is not None and (root / "src" / "fips202" / "fips202.c").exists():
            oracle.build(ref=True)
        else:
            pytest.skip("reference fips202.c not built (set CUDIL_REF_ROOT to the reference tree)")
    ref = ctypes.CDLL(str(oracle.REF_LIB))
    rng = random.Random(11)
    for n in [0, 3, 136, 168, 333, 2000]:
        data = bytes(rng.getrandbits(8) for _ in range(n))
        for outlen in [32, 64, 840]:
            a = ctypes.create_string_buffer(outlen)
            ref.shake128(a, ctypes.c_size_t(outlen), data, ctypes.c_size_t(n))
            assert oracle.shake128(data, outlen) == a.raw
            ref.shake256(a, ctypes.c_size_t(outlen), data, ctypes.c_size_t(n))
            assert oracle.shake256(data, outlen) == a.raw


def test_ntt_roundtrip_and_product(oracle):
    """invNTT(NTT(a) o mont^2-ish) identities: NTT->invNTT multiplies by 2^32 mod q (tomont)."""
    q = 8380417
    rng = np.random.default_rng(3)
    a = rng.integers(0, q, 256, dtype=np.int64).astype(np.int32)
    r = oracle.invntt_tomont(oracle.ntt(a)).astype(np.int64)
    mont = (1 << 32) % q
    assert np.all((r - a.astype(np.int64) * mont) % q == 0)
    # schoolbook negacyclic product vs NTT product: invNTT(NTT(a) o NTT(b)) = a*b (mod q, x^256+1)
    b = rng.integers(-4, 5, 256, dtype=np.int64).astype(np.int32)
    ah, bh = oracle.ntt(a), oracle.ntt(b)
    prod = oracle.ntt_mul_batch(a[None, :], bh[None, :])[0].astype(np.int64)
    ref = np.zeros(256, dtype=object)
    for i in range(256):
        for j in range(256):
            k = i + j
            v = int(a[i]) * int(b[j])
            if k >= 256:
                ref[k - 256] -= v
            else:
                ref[k] += v
    ref = np.array([int(x) % q for x in ref], dtype=np.int64)
    assert np.all((prod - ref) % q == 0)


@pytest.mark.parametrize("mode", MODES)
def test_oracle_negative_cases(oracle, mode):
    p = oracle.params(mode)
    m = oracle.messages_from_ctr(6, 48)
    pk, sk = oracle.keypair_batch(mode, 6, rand_index=100)
    sig = oracle.sign_batch(mode, m, sk)
    assert np.all(oracle.verify_batch(mode, sig, m, pk) == 0)
    bad = sig.copy()
    bad[0, 5] ^= 1          # c~
    bad[1, 100] ^= 0x10     # z
    bad[2, p.sig_bytes - 1] = 0xFF  # omega count out of range
    m2 = m.copy()
    m2[3, 0] ^= 1
    ret = oracle.verify_batch(mode, bad, m2, pk)
    assert list(ret[:4]) == [-1, -1, -1, -1]
    assert np.all(oracle.verify_batch(mode, sig, m, pk, siglen=p.sig_bytes - 1) == -1)


@pytest.mark.parametrize("mode", [2, 3, 5])
def test_oracle_parse_checks(oracle, mode):
    """The parse checks accept genuine encodings and flag malformed hints / z / eta fields; a
    flagged signature never verifies."""
    p = oracle.params(mode)
    pk, sk = oracle.keypair_batch(mode, 6, rand_index=77 + mode)
    m = oracle.messages_from_ctr(6, 32)
    sig = oracle.sign_batch(mode, m, sk)
    assert np.all(oracle.sig_check(mode, sig) == 0) and np.all(oracle.sk_check(mode, sk) == 0)
    h0 = 32 + p.l * p.polyz_packed
    bad = sig.copy()
    bad[0, h0 + p.omega + p.k - 1] = p.omega + 1
    bad[1, 32:35] = 0
    st = oracle.sig_check(mode, bad)
    assert st[0] & 1 and st[1] & 2
    assert np.all(oracle.verify_batch(mode, bad[:2], m[:2], pk[:2]) == -1)
    bsk = sk.copy()
    bsk[3, 96] = 0xFF
    assert oracle.sk_check(mode, bsk)[3] == 1


def test_reference_xor_ballots_accept_noncanonical_hints(oracle):
    """The reference's XOR-combined hint ballots (src/verify.cu:66, :85) accept re-encoded valid
    signatures that the scheme's checks -- the oracle's ora_verify and the CUDA library -- reject.
    This pins the one place where verification deliberately differs from the reference."""
    from hint_cases import all_cases
    for label, mode, pk, m, sig, bad in all_cases(oracle):
        assert oracle.verify_batch(mode, sig[None], m[None], pk[None])[0] == 0, label
        assert oracle.verify_xor_ballots(mode, sig, m.tobytes(), pk) == 0, label
        # the re-encoding keeps the decoded hints: the reference's form still accepts it ...
        assert oracle.verify_xor_ballots(mode, bad, m.tobytes(), pk) == 0, label
        assert oracle.hint_check(mode, bad, xor_lanes=True)[0] == 0, label
        # ... while the scheme's form rejects it
        assert oracle.verify_batch(mode, bad[None], m[None], pk[None])[0] == -1, label
        assert oracle.hint_check(mode, bad)[0] == 1 and oracle.sig_check(mode, bad)[0] & 1, label
    # a single violation is rejected by both forms
    pk, m, sig, bad = all_cases(oracle)[0][2:]
    p = oracle.params(2)
    one = bad.copy()
    one[32 + p.l * p.polyz_packed + int(sig[32 + p.l * p.polyz_packed + p.omega + p.k - 1]) + 32] = 0
    assert oracle.verify_xor_ballots(2, one, m.tobytes(), pk) == -1


def test_first_call_on_many_threads_is_deterministic():
    """The oracle's tables are ready before any caller thread runs: a fresh process whose first
    oracle call is a batch on several OpenMP threads gets the same keys as a single thread."""
    import subprocess
    import sys
    from pathlib import Path
    code = ("import sys; sys.path.insert(0, %r)\n"
            "import numpy as np\n"
            "from oracle import pyoracle as O\n"
            "pk, sk = O.keypair_batch(2, 512, 0, 8)\n"
            "pk1, sk1 = O.keypair_seeds(2, O.seeds_from_ctr(512), 1)\n"
            "assert np.array_equal(pk, pk1) and np.array_equal(sk, sk1)\n" % str(Path(__file__).resolve().parents[1]))
    for _ in range(3):
        subprocess.run([sys.executable, "-c", code], check=True)


def test_derive_rhoprime_matches_shake256(oracle):
    """The oracle's randomized-signing seed derivation against Python's own SHAKE256."""
    seed = bytes(range(7, 39))
    for counter in (0, 1, 2**32 - 1, 2**64 - 3):
        got = oracle.derive_rhoprime(seed, counter, 3)
        for i in range(3):
            c = (counter + i) % 2**64
            assert got[i].tobytes() == hashlib.shake_256(seed + c.to_bytes(8, "little")).digest(64)
