"""ctypes binding of the CPU oracle ``oracle/liboracle.so`` (test infrastructure only).

The oracle is a C restatement of the reference's algorithm (see oracle/dilithium.c), pinned to
the reference's test-vector digests.  It is the checker for the CUDA library and the timed CPU
baseline; nothing in the product calls it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_char_p, c_int, c_int32, c_long, c_size_t, c_uint8, c_uint16, c_uint64, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libref_fips202.so"


def ref_root() -> Path | None:
    """Root of the reference source tree, from CUDIL_REF_ROOT (unset: no reference build)."""
    r = os.environ.get("CUDIL_REF_ROOT")
    return Path(r) if r else None


def build(ref: bool = True) -> None:
    """make -C oracle (and the reference's own fips202.c into oracle/_ref when CUDIL_REF_ROOT names
    a reference tree that holds it)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    root = ref_root()
    if ref and root is not None and (root / "src" / "fips202" / "fips202.c").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF_ROOT={root}"], check=True)


class ora_params(ctypes.Structure):
    _fields_ = [(n, c_int) for n in (
        "mode", "k", "l", "eta", "tau", "beta", "gamma1", "gamma2", "omega",
        "polyz_packed", "polyw1_packed", "polyeta_packed", "pk_bytes", "sk_bytes", "sig_bytes")]


def _load():
    if not LIB.exists():
        build(ref=False)
    lib = ctypes.CDLL(str(LIB))
    P8 = c_void_p
    sig = {
        "ora_params_get": (c_int, [c_int, POINTER(ora_params)]),
        "ora_shake128": (None, [P8, c_size_t, P8, c_size_t]),
        "ora_shake256": (None, [P8, c_size_t, P8, c_size_t]),
        "ora_keypair_from_seed": (c_int, [c_int, P8, P8, P8]),
        "ora_sign": (c_int, [c_int, P8, P8, c_size_t, P8, POINTER(c_int)]),
        "ora_sign_rhoprime": (c_int, [c_int, P8, P8, c_size_t, P8, P8, POINTER(c_int)]),
        "ora_sig_check": (c_int, [c_int, P8]),
        "ora_hint_check": (c_int, [c_int, P8, c_int]),
        "ora_derive_rhoprime": (None, [P8, P8, c_uint64, c_size_t]),
        "ora_verify_xor_ballots": (c_int, [c_int, P8, c_size_t, P8, c_size_t, P8]),
        "ora_sk_check": (c_int, [c_int, P8]),
        "ora_verify": (c_int, [c_int, P8, c_size_t, P8, c_size_t, P8]),
        "ora_seed_from_ctr": (None, [P8, c_uint64]),
        "ora_keypair_batch": (c_int, [c_int, P8, P8, c_size_t, c_uint64, c_int]),
        "ora_keypair_seeds_batch": (c_int, [c_int, P8, P8, P8, c_size_t, c_int]),
        "ora_sign_batch": (c_int, [c_int, P8, c_size_t, P8, c_size_t, P8, P8, c_size_t, c_size_t, c_int, P8]),
        "ora_verify_batch": (c_int, [c_int, P8, P8, c_size_t, c_size_t, P8, c_size_t, P8, P8, c_size_t, c_size_t,
                                     c_int]),
        "ora_ntt": (None, [P8]),
        "ora_invntt_tomont": (None, [P8]),
        "ora_ntt_mul_batch": (None, [P8, P8, c_size_t, c_int]),
        "ora_expand_a": (None, [c_int, P8, P8]),
        "ora_expand_mask": (None, [c_int, P8, P8, c_uint16]),
        "ora_challenge": (None, [c_int, P8, P8]),
        "ora_tvecs": (c_long, [c_int, c_size_t, P8, c_size_t, c_int]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def params(mode: int) -> ora_params:
    p = ora_params()
    assert lib.ora_params_get(mode, ctypes.byref(p)) == 0
    return p


def shake128(data: bytes, outlen: int) -> bytes:
    out = ctypes.create_string_buffer(outlen)
    lib.ora_shake128(out, outlen, data, len(data))
    return out.raw


def shake256(data: bytes, outlen: int) -> bytes:
    out = ctypes.create_string_buffer(outlen)
    lib.ora_shake256(out, outlen, data, len(data))
    return out.raw


def seeds_from_ctr(n: int, rand_index: int = 0) -> np.ndarray:
    """Key seeds of the reference's keypair kernel: SHAKE128(le64(rand_index + 2i + 1))[0:32]."""
    out = np.zeros((n, 32), dtype=np.uint8)
    for i in range(n):
        lib.ora_seed_from_ctr(_p(out[i]), rand_index + 2 * i + 1)
    return out


def messages_from_ctr(n: int, mlen: int = 32) -> np.ndarray:
    """Messages of the reference's test: SHAKE128(le64(2i))[0:mlen]."""
    return np.stack([np.frombuffer(shake128((2 * i).to_bytes(8, "little"), mlen), dtype=np.uint8)
                     for i in range(n)]) if n else np.zeros((0, mlen), np.uint8)


def keypair_batch(mode: int, n: int, rand_index: int = 0, nthreads: int = 0):
    p = params(mode)
    pk = np.zeros((n, p.pk_bytes), np.uint8)
    sk = np.zeros((n, p.sk_bytes), np.uint8)
    assert lib.ora_keypair_batch(mode, _p(pk), _p(sk), n, rand_index, nthreads) == 0
    return pk, sk


def keypair_seeds(mode: int, seeds: np.ndarray, nthreads: int = 0):
    p = params(mode)
    seeds = np.ascontiguousarray(seeds, dtype=np.uint8)
    n = seeds.shape[0]
    pk = np.zeros((n, p.pk_bytes), np.uint8)
    sk = np.zeros((n, p.sk_bytes), np.uint8)
    assert lib.ora_keypair_seeds_batch(mode, _p(pk), _p(sk), _p(seeds), n, nthreads) == 0
    return pk, sk


def sign_batch(mode: int, m: np.ndarray, sk: np.ndarray, mlens=None, nthreads: int = 0, return_attempts=False):
    """m: (n, stride) uint8 with per-item lengths mlens (default: full rows)."""
    p = params(mode)
    m = np.ascontiguousarray(m, dtype=np.uint8)
    sk = np.ascontiguousarray(sk, dtype=np.uint8)
    n, stride = m.shape
    ml = np.full(n, stride, np.uint64) if mlens is None else np.ascontiguousarray(mlens, dtype=np.uint64)
    sig = np.zeros((n, p.sig_bytes), np.uint8)
    att = np.zeros(n, np.int32)
    assert lib.ora_sign_batch(mode, _p(sig), p.sig_bytes, _p(m), stride, _p(ml), _p(sk), p.sk_bytes, n, nthreads,
                              _p(att)) == 0
    return (sig, att) if return_attempts else sig


def sign_rhoprime(mode: int, m: bytes, sk: np.ndarray, rhoprime: bytes) -> np.ndarray:
    """Randomized signing with a given rho' (64 bytes) instead of SHAKE256(K || mu)
    (reference src/api.cu:143-148)."""
    p = params(mode)
    sig = np.zeros(p.sig_bytes, np.uint8)
    mb = np.frombuffer(bytes(m) + b"\0", np.uint8)
    skb = np.ascontiguousarray(sk, dtype=np.uint8).reshape(-1)
    rp = np.frombuffer(bytes(rhoprime), np.uint8)
    assert rp.size == 64
    att = ctypes.c_int(0)
    assert lib.ora_sign_rhoprime(mode, _p(sig), _p(mb), len(m), _p(skb), _p(rp), ctypes.byref(att)) == 0
    return sig


def derive_rhoprime(seed: bytes, counter: int, n: int) -> np.ndarray:
    """(n, 64) randomized-signing seeds: rho'_i = SHAKE256(seed || le64(counter + i), 64)."""
    out = np.zeros((max(n, 1), 64), np.uint8)
    s = np.frombuffer(bytes(seed), np.uint8)
    assert s.size == 32
    lib.ora_derive_rhoprime(_p(out), _p(s), counter, n)
    return out[:n]


def sig_check(mode: int, sig: np.ndarray) -> np.ndarray:
    """Per-signature parse status: bit 0 bad hint encoding, bit 1 z out of range."""
    sig = np.ascontiguousarray(sig, dtype=np.uint8).reshape(-1, params(mode).sig_bytes)
    return np.array([lib.ora_sig_check(mode, _p(np.ascontiguousarray(r))) for r in sig], dtype=np.int32)


def hint_check(mode: int, sig: np.ndarray, xor_lanes: bool = False) -> np.ndarray:
    """Per-signature hint-encoding status (0 accepted, 1 rejected).  xor_lanes=True evaluates the
    checks as the reference kernel does (lane ballots combined with XOR, src/verify.cu:66, :85)."""
    sig = np.ascontiguousarray(sig, dtype=np.uint8).reshape(-1, params(mode).sig_bytes)
    return np.array([lib.ora_hint_check(mode, _p(np.ascontiguousarray(r)), int(xor_lanes)) for r in sig],
                    dtype=np.int32)


def verify_xor_ballots(mode: int, sig: np.ndarray, m: bytes, pk: np.ndarray) -> int:
    """One verification with the reference kernel's XOR-combined hint ballots (0 valid, -1 not)."""
    s = np.ascontiguousarray(sig, dtype=np.uint8).reshape(-1)
    mb = np.frombuffer(bytes(m) + b"\0", np.uint8)
    k = np.ascontiguousarray(pk, dtype=np.uint8).reshape(-1)
    return int(lib.ora_verify_xor_ballots(mode, _p(s), s.size, _p(mb), len(m), _p(k)))


def sk_check(mode: int, sk: np.ndarray) -> np.ndarray:
    """Per-key parse status: bit 0 an s1/s2 eta field out of range."""
    sk = np.ascontiguousarray(sk, dtype=np.uint8).reshape(-1, params(mode).sk_bytes)
    return np.array([lib.ora_sk_check(mode, _p(np.ascontiguousarray(r))) for r in sk], dtype=np.int32)


def verify_batch(mode: int, sig: np.ndarray, m: np.ndarray, pk: np.ndarray, mlens=None, siglen=None,
                 nthreads: int = 0) -> np.ndarray:
    p = params(mode)
    sig = np.ascontiguousarray(sig, dtype=np.uint8)
    m = np.ascontiguousarray(m, dtype=np.uint8)
    pk = np.ascontiguousarray(pk, dtype=np.uint8)
    n, stride = m.shape
    ml = np.full(n, stride, np.uint64) if mlens is None else np.ascontiguousarray(mlens, dtype=np.uint64)
    ret = np.zeros(n, np.int32)
    lib.ora_verify_batch(mode, _p(ret), _p(sig), sig.shape[1], p.sig_bytes if siglen is None else siglen, _p(m),
                         stride, _p(ml), _p(pk), pk.shape[1], n, nthreads)
    return ret


def ntt_mul_batch(a: np.ndarray, b: np.ndarray, nthreads: int = 0) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.int32).copy()
    b = np.ascontiguousarray(b, dtype=np.int32)
    lib.ora_ntt_mul_batch(_p(a), _p(b), a.shape[0], nthreads)
    return a


def ntt(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.int32).copy()
    lib.ora_ntt(_p(a))
    return a


def invntt_tomont(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.int32).copy()
    lib.ora_invntt_tomont(_p(a))
    return a


def tvecs(mode: int, nvectors: int = 10000, nthreads: int = 0) -> bytes:
    """The reference's tvecs<mode> file for the first nvectors items."""
    buf = ctypes.create_string_buffer(nvectors * 400 + 64)
    n = lib.ora_tvecs(mode, nvectors, buf, len(buf), nthreads)
    assert n > 0
    return buf.raw[:n]


def tvecs_from_outputs(m: np.ndarray, pk: np.ndarray, sk: np.ndarray, sig: np.ndarray, ret: np.ndarray) -> bytes:
    """Formats outputs (from any implementation) exactly as tests/test_vectors.cu:177-209 does."""
    lines = []
    for i in range(len(ret)):
        if ret[i]:
            lines.append(f"Signature verification failed! {i}\n")
    for i in range(m.shape[0]):
        lines.append(f"count = {i}\n")
        lines.append("m = " + m[i].tobytes().hex() + "\n")
        lines.append("pk = " + shake256(pk[i].tobytes(), 32).hex() + "\n")
        lines.append("sk = " + shake256(sk[i].tobytes(), 32).hex() + "\n")
        lines.append("sig = " + shake256(sig[i].tobytes(), 32).hex() + "\n")
    return "".join(lines).encode()
