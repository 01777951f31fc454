"""Host-side mirror of the reference's public API (include/api.cuh:27-63) over the CUDA library.

``Dilithium(mode)`` plays the role of one of the reference's per-mode libraries
(cuDilithium2/3/5): ``crypto_sign_keypair``, ``crypto_sign_signature`` and ``crypto_sign_verify``
take the same arguments in the same order (buffers as torch tensors: pinned host tensors for
the host arrays, CUDA tensors for the pools and LUT device arrays) and keep the reference's
behaviour: keypair and verify are asynchronous on ``stream``, sign synchronizes once per
rejection round, verify with a wrong ``siglen`` fills ``ret`` with -1 without touching the GPU.

Convenience wrappers (``keypair``, ``sign``, ``verify``) allocate pools themselves the way the
reference's tests do (tests/test_vectors.cu:62-166) and return numpy arrays.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import check, lib

PITCH_ALIGN = 512  # what cudaMallocPitch returns on current GPUs


def _ptr(t) -> int | None:
    if t is None:
        return None
    if isinstance(t, int):
        return t
    return t.data_ptr()


def _stream_ptr(stream) -> int | None:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def pitch_for(row_bytes: int) -> int:
    return (row_bytes + PITCH_ALIGN - 1) // PITCH_ALIGN * PITCH_ALIGN


def alloc_pool(row_bytes: int, rows: int, device="cuda") -> tuple[torch.Tensor, int]:
    """Pitched device pool (the cudaMallocPitch of the reference's callers)."""
    pitch = pitch_for(row_bytes)
    return torch.empty((max(rows, 1), pitch), dtype=torch.uint8, device=device), pitch


def pinned(nbytes: int) -> torch.Tensor:
    return torch.empty(max(nbytes, 1), dtype=torch.uint8, pin_memory=True)


class TaskLut:
    """The reference's task_lut (include/api.cuh:41-49): a per-item sign LUT on the host plus
    exec/done/copy arrays of exec_threshold entries on the host (pinned) and the device."""

    def __init__(self, batch_size: int, exec_threshold: int, device="cuda"):
        self.batch_size = batch_size
        self.exec_threshold = exec_threshold
        self._sign_lut = (_lib.cudil_sign_lut_element * max(batch_size, 1))()
        esz = ctypes.sizeof(_lib.cudil_copy_lut_element)
        self.h_exec = pinned(4 * exec_threshold)
        self.h_done = pinned(exec_threshold)
        self.h_copy = pinned(esz * exec_threshold)
        self.d_exec = torch.empty(4 * exec_threshold, dtype=torch.uint8, device=device)
        self.d_done = torch.empty(exec_threshold, dtype=torch.uint8, device=device)
        self.d_copy = torch.empty(esz * exec_threshold, dtype=torch.uint8, device=device)
        self.c = _lib.cudil_task_lut(
            ctypes.cast(self._sign_lut, ctypes.POINTER(_lib.cudil_sign_lut_element)), batch_size,
            _ptr(self.h_exec), _ptr(self.h_done), _ptr(self.h_copy),
            _ptr(self.d_exec), _ptr(self.d_done), _ptr(self.d_copy))

    def nonces(self) -> np.ndarray:
        """Attempts issued per item in the last call (the reference's sign_lut[i].nonce)."""
        return np.array([e.nonce for e in self._sign_lut[: self.batch_size]], dtype=np.int64)


@dataclass
class Dilithium:
    """One parameter set (2, 3 or 5), like the reference's cuDilithium<mode> library."""

    mode: int

    def __post_init__(self):
        p = _lib.params(self.mode)
        self.params = p
        self.CRYPTO_PUBLICKEYBYTES = p.pk_bytes
        self.CRYPTO_SECRETKEYBYTES = p.sk_bytes
        self.CRYPTO_BYTES = p.sig_bytes

    # -------------------------------------------------------------- row sizes
    def keypair_row_bytes(self) -> int:
        return lib.cudil_keypair_row_bytes(self.mode)

    def sign_row_bytes(self, mlen: int) -> int:
        return lib.cudil_sign_row_bytes(self.mode, mlen)

    def sign_temp_row_bytes(self) -> int:
        return lib.cudil_sign_temp_row_bytes(self.mode)

    def verify_row_bytes(self, mlen: int) -> int:
        return lib.cudil_verify_row_bytes(self.mode, mlen)

    # -------------------------------------------------------------- reference API
    def crypto_sign_keypair(self, pk, sk, d_keypair_mem_pool, keypair_mem_pool_pitch, batch_size=1, stream=None,
                            rand_index=0) -> int:
        rc = lib.cudil_keypair(self.mode, _ptr(pk), _ptr(sk), _ptr(d_keypair_mem_pool), keypair_mem_pool_pitch,
                               batch_size, _stream_ptr(stream), rand_index)
        check(rc, "crypto_sign_keypair")
        return 0

    def crypto_sign_keypair_from_seed(self, pk, sk, seeds, d_keypair_mem_pool, keypair_mem_pool_pitch, batch_size=1,
                                      stream=None) -> int:
        rc = lib.cudil_keypair_from_seed(self.mode, _ptr(pk), _ptr(sk), _ptr(seeds), _ptr(d_keypair_mem_pool),
                                         keypair_mem_pool_pitch, batch_size, _stream_ptr(stream))
        check(rc, "crypto_sign_keypair_from_seed")
        return 0

    def crypto_sign_signature(self, sig, sig_pitch, siglen, m, m_pitch, mlen, sk, d_sign_mem_pool,
                              d_sign_mem_pool_pitch, d_temp_mem_pool, d_temp_mem_pool_pitch, lut: TaskLut,
                              exec_threshold, batch_size=1, stream=None) -> int:
        sl = ctypes.c_size_t(0)
        rc = lib.cudil_sign(self.mode, _ptr(sig), sig_pitch, ctypes.byref(sl), _ptr(m), m_pitch, mlen, _ptr(sk),
                            _ptr(d_sign_mem_pool), d_sign_mem_pool_pitch, _ptr(d_temp_mem_pool),
                            d_temp_mem_pool_pitch, ctypes.byref(lut.c), exec_threshold, batch_size,
                            _stream_ptr(stream))
        check(rc, "crypto_sign_signature")
        if isinstance(siglen, list):
            siglen[:] = [sl.value]
        return 0

    def crypto_sign_verify(self, ret, sig, sig_pitch, siglen, m, m_pitch, mlen, pk, d_verify_mem_pool,
                           verify_mem_pool_pitch, batch_size=1, stream=None) -> None:
        rc = lib.cudil_verify(self.mode, _ptr(ret), _ptr(sig), sig_pitch, siglen, _ptr(m), m_pitch, mlen, _ptr(pk),
                              _ptr(d_verify_mem_pool), verify_mem_pool_pitch, batch_size, _stream_ptr(stream))
        check(rc, "crypto_sign_verify")

    # -------------------------------------------------------------- conveniences
    def keypair(self, n: int, rand_index: int = 0, seeds: np.ndarray | None = None):
        pool, pitch = alloc_pool(self.keypair_row_bytes(), n)
        pk = pinned(n * self.CRYPTO_PUBLICKEYBYTES)
        sk = pinned(n * self.CRYPTO_SECRETKEYBYTES)
        if seeds is not None:
            s = pinned(n * 32)
            s.numpy()[: n * 32] = np.ascontiguousarray(seeds, dtype=np.uint8).reshape(-1)
            self.crypto_sign_keypair_from_seed(pk, sk, s, pool, pitch, n)
        else:
            self.crypto_sign_keypair(pk, sk, pool, pitch, n, None, rand_index)
        torch.cuda.synchronize()
        return (pk.numpy()[: n * self.CRYPTO_PUBLICKEYBYTES].reshape(n, self.CRYPTO_PUBLICKEYBYTES).copy(),
                sk.numpy()[: n * self.CRYPTO_SECRETKEYBYTES].reshape(n, self.CRYPTO_SECRETKEYBYTES).copy())

    def sign(self, m: np.ndarray, sk: np.ndarray, exec_threshold: int = 2048, return_lut: bool = False,
             rhoprime: np.ndarray | None = None):
        """rhoprime: optional (n, 64) random seeds for randomized signing (cudil_sign_randomized);
        None = deterministic signing."""
        m = np.ascontiguousarray(m, dtype=np.uint8)
        n, mlen = m.shape
        pool, sp = alloc_pool(self.sign_row_bytes(mlen), n)
        tpool, tp = alloc_pool(self.sign_temp_row_bytes(), exec_threshold)
        lut = TaskLut(n, exec_threshold)
        hm = pinned(m.size)
        hm.numpy()[: m.size] = m.reshape(-1)
        hsk = pinned(n * self.CRYPTO_SECRETKEYBYTES)
        hsk.numpy()[: n * self.CRYPTO_SECRETKEYBYTES] = np.ascontiguousarray(sk, dtype=np.uint8).reshape(-1)
        hsig = pinned(n * self.CRYPTO_BYTES)
        siglen = [0]
        if rhoprime is None:
            self.crypto_sign_signature(hsig, self.CRYPTO_BYTES, siglen, hm, mlen, mlen, hsk, pool, sp, tpool, tp, lut,
                                       exec_threshold, n)
        else:
            hr = pinned(n * 64)
            hr.numpy()[: n * 64] = np.ascontiguousarray(rhoprime, dtype=np.uint8).reshape(-1)
            sl = ctypes.c_size_t(0)
            check(lib.cudil_sign_randomized(self.mode, _ptr(hsig), self.CRYPTO_BYTES, ctypes.byref(sl), _ptr(hm), mlen,
                                            mlen, _ptr(hsk), _ptr(hr), 64, _ptr(pool), sp, _ptr(tpool), tp,
                                            ctypes.byref(lut.c), exec_threshold, n, None), "cudil_sign_randomized")
        torch.cuda.synchronize()
        sig = hsig.numpy()[: n * self.CRYPTO_BYTES].reshape(n, self.CRYPTO_BYTES).copy()
        return (sig, lut) if return_lut else sig

    def crypto_sign(self, m: np.ndarray, sk: np.ndarray, exec_threshold: int = 2048) -> np.ndarray:
        """Signed messages sm = sig || m for every row of m (cudil_crypto_sign)."""
        m = np.ascontiguousarray(m, dtype=np.uint8)
        n, mlen = m.shape
        smb = self.CRYPTO_BYTES + mlen
        pool, sp = alloc_pool(self.sign_row_bytes(mlen), n)
        tpool, tp = alloc_pool(self.sign_temp_row_bytes(), exec_threshold)
        lut = TaskLut(n, exec_threshold)
        hm = pinned(max(m.size, 1))
        hm.numpy()[: m.size] = m.reshape(-1)
        hsk = pinned(n * self.CRYPTO_SECRETKEYBYTES)
        hsk.numpy()[: n * self.CRYPTO_SECRETKEYBYTES] = np.ascontiguousarray(sk, dtype=np.uint8).reshape(-1)
        hsm = pinned(n * smb)
        smlen = ctypes.c_size_t(0)
        check(lib.cudil_crypto_sign(self.mode, _ptr(hsm), smb, ctypes.byref(smlen), _ptr(hm), mlen, mlen, _ptr(hsk),
                                    _ptr(pool), sp, _ptr(tpool), tp, ctypes.byref(lut.c), exec_threshold, n, None),
              "cudil_crypto_sign")
        torch.cuda.synchronize()
        assert smlen.value == smb
        return hsm.numpy()[: n * smb].reshape(n, smb).copy()

    def crypto_sign_open(self, sm: np.ndarray, pk: np.ndarray):
        """(messages, ret) for every row of sm (cudil_crypto_sign_open); invalid rows give ret -1
        and a zeroed message."""
        sm = np.ascontiguousarray(sm, dtype=np.uint8)
        n, smlen = sm.shape
        mlen = max(smlen - self.CRYPTO_BYTES, 0)
        pool, pitch = alloc_pool(self.verify_row_bytes(mlen), n)
        hsm = pinned(max(sm.size, 1))
        hsm.numpy()[: sm.size] = sm.reshape(-1)
        hpk = pinned(n * self.CRYPTO_PUBLICKEYBYTES)
        hpk.numpy()[: n * self.CRYPTO_PUBLICKEYBYTES] = np.ascontiguousarray(pk, dtype=np.uint8).reshape(-1)
        hm = pinned(max(n * mlen, 1))
        hret = pinned(n * 4)
        ml = ctypes.c_size_t(12345)
        check(lib.cudil_crypto_sign_open(self.mode, _ptr(hm), max(mlen, 1), ctypes.byref(ml), _ptr(hret), _ptr(hsm),
                                         smlen, smlen, _ptr(hpk), _ptr(pool), pitch, n, None), "cudil_crypto_sign_open")
        ret = hret.numpy()[: n * 4].view(np.int32).copy()
        return hm.numpy()[: n * mlen].reshape(n, mlen).copy(), ret, ml.value

    def sig_check(self, sig: np.ndarray, sig_pitch: int | None = None) -> np.ndarray:
        """Parse step on the GPU (cudil_sig_check): per signature, bit 0 = bad hint encoding,
        bit 1 = a z coefficient out of range."""
        sig = np.ascontiguousarray(sig, dtype=np.uint8)
        n = sig.shape[0]
        pitch = sig_pitch or sig.shape[1]
        d_sig = torch.from_numpy(sig.reshape(-1)).cuda()
        d_st = torch.full((max(n, 1),), -7, dtype=torch.int32, device="cuda")
        check(lib.cudil_sig_check(self.mode, _ptr(d_st), _ptr(d_sig), pitch, n, None), "cudil_sig_check")
        torch.cuda.synchronize()
        return d_st.cpu().numpy()[:n]

    def sk_check(self, sk: np.ndarray) -> np.ndarray:
        """Parse step on the GPU (cudil_sk_check): 1 where an s1/s2 eta field is out of range."""
        sk = np.ascontiguousarray(sk, dtype=np.uint8)
        n = sk.shape[0]
        d_sk = torch.from_numpy(sk.reshape(-1)).cuda()
        d_st = torch.full((max(n, 1),), -7, dtype=torch.int32, device="cuda")
        check(lib.cudil_sk_check(self.mode, _ptr(d_st), _ptr(d_sk), n, None), "cudil_sk_check")
        torch.cuda.synchronize()
        return d_st.cpu().numpy()[:n]

    def verify(self, sig: np.ndarray, m: np.ndarray, pk: np.ndarray, siglen: int | None = None) -> np.ndarray:
        m = np.ascontiguousarray(m, dtype=np.uint8)
        n, mlen = m.shape
        pool, pitch = alloc_pool(self.verify_row_bytes(mlen), n)
        hsig = pinned(n * self.CRYPTO_BYTES)
        hsig.numpy()[: n * self.CRYPTO_BYTES] = np.ascontiguousarray(sig, dtype=np.uint8).reshape(-1)
        hm = pinned(m.size)
        hm.numpy()[: m.size] = m.reshape(-1)
        hpk = pinned(n * self.CRYPTO_PUBLICKEYBYTES)
        hpk.numpy()[: n * self.CRYPTO_PUBLICKEYBYTES] = np.ascontiguousarray(pk, dtype=np.uint8).reshape(-1)
        ret = torch.empty(max(n, 1), dtype=torch.int32, pin_memory=True)
        self.crypto_sign_verify(ret, hsig, self.CRYPTO_BYTES, self.CRYPTO_BYTES if siglen is None else siglen, hm,
                                mlen, mlen, hpk, pool, pitch, n)
        torch.cuda.synchronize()
        return ret.numpy()[:n].copy()


def derive_rhoprime(seed: bytes, counter: int, n: int, stream=None) -> torch.Tensor:
    """(n, 64) uint8 CUDA tensor of randomized-signing seeds, row i = SHAKE256(seed || le64(counter + i),
    64), derived on the device from one 32-byte seed (cudil_derive_rhoprime)."""
    seed = bytes(seed)
    if len(seed) != 32:
        raise ValueError("seed must be 32 bytes")
    out = torch.empty((max(n, 1), 64), dtype=torch.uint8, device="cuda")
    check(lib.cudil_derive_rhoprime(_ptr(out), 64, seed, counter, n, _stream_ptr(stream)), "cudil_derive_rhoprime")
    return out[:n]


def ntt_mul(a: torch.Tensor, b: torch.Tensor, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """out[p] = invNTT(NTT(a[p]) o b[p]) for int32 CUDA tensors of shape (npolys, 256)."""
    assert a.is_cuda and b.is_cuda and a.dtype == torch.int32 and b.dtype == torch.int32
    assert a.shape == b.shape and a.shape[-1] == 256 and a.is_contiguous() and b.is_contiguous()
    if out is None:
        out = torch.empty_like(a)
    n = a.numel() // 256
    check(lib.cudil_ntt_mul(_ptr(a), _ptr(b), _ptr(out), n, _stream_ptr(stream)), "cudil_ntt_mul")
    return out
