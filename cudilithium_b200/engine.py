"""Fused engine: per-key resident caches + one persistent, graph-launched kernel per batch.

Python host side of the ``cudil_engine_*`` C ABI (include/cudilithium.h).  An ``Engine`` wraps one
engine of one parameter set on the current CUDA device; an ``EnginePipeline`` runs a stream of
batches over several engines on their own streams.  Messages are packed into one device buffer at
8-byte aligned offsets (``pack_messages``).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import check, lib


def pack_messages(msgs: list[bytes] | np.ndarray, device="cuda"):
    """Packs messages into one device buffer; returns (buffer, offsets, lengths) with every
    offset a multiple of 8 (the engine reads message lanes as aligned 8-byte words)."""
    if isinstance(msgs, np.ndarray):
        msgs = [bytes(r) for r in msgs]
    lens = np.array([len(m) for m in msgs], dtype=np.uint32)
    offs = np.zeros(len(msgs), dtype=np.uint64)
    pos = 0
    for i, m in enumerate(msgs):
        offs[i] = pos
        pos += (len(m) + 7) // 8 * 8
    host = np.zeros(max(pos, 8) + 8, dtype=np.uint8)
    for i, m in enumerate(msgs):
        host[int(offs[i]): int(offs[i]) + len(m)] = np.frombuffer(m, dtype=np.uint8)
    return torch.from_numpy(host).to(device), offs, lens


class Engine:
    """One cudil_engine (one parameter set, current device)."""

    def __init__(self, mode: int, max_keys: int, max_items: int, threads: int = 0, budget_bytes: int = 0,
                 spec_slots: int = 0):
        """threads / spec_slots = 0 take the autotuned settings for this GPU (autotune.tuned)."""
        from .autotune import tuned
        self.mode = mode
        self.params = _lib.params(mode)
        self.max_keys, self.max_items = max_keys, max_items
        t = tuned(mode)
        threads = threads or t["threads"]
        h = ctypes.c_void_p()
        check(lib.cudil_engine_create(ctypes.byref(h), mode, max_keys, max_items, threads, budget_bytes),
              "cudil_engine_create")
        self.h = h
        self.set_sign_kernel(t.get("sign_kernel", 0))
        self.set_spec_slots(spec_slots or t["spec_slots"])

    def close(self):
        if self.h:
            lib.cudil_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def device_bytes(self) -> int:
        return lib.cudil_engine_device_bytes(self.h)

    def set_sign_kernel(self, variant: int):
        """0 phased persistent signer; 1..4 asynchronous with (threads, slots) per block of
        (256, 64), (512, 128), (640, 160), (768, 192); 5 phased with one wide block per SM (512
        threads, 384 for Dilithium5); see cudil_engine_set_sign_kernel."""
        check(lib.cudil_engine_set_sign_kernel(self.h, variant), "set_sign_kernel")
        self.sign_kernel = variant

    def set_large_batch(self, min_items: int, variant: int = 5, spec_slots: int = 128):
        """Signer for batches of at least min_items items (0 = off); see cudil_engine_set_large_batch."""
        check(lib.cudil_engine_set_large_batch(self.h, min_items, variant, spec_slots), "set_large_batch")

    def last_jobs(self) -> dict:
        """Asynchronous signer job profile of the last batch: {job: (cycles summed over warps, count)}."""
        v = (ctypes.c_ulonglong * 12)()
        check(lib.cudil_engine_last_jobs(self.h, v), "last_jobs")
        names = ("reject", "w", "challenge", "mask", "claim", "idle")
        return {k: (v[i], v[6 + i]) for i, k in enumerate(names)}

    def set_spec_slots(self, slots: int):
        """Per-block target of signing attempts in flight; see cudil_engine_set_spec_slots."""
        check(lib.cudil_engine_set_spec_slots(self.h, slots), "set_spec_slots")

    def info(self) -> dict:
        m, t, sb, vb = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        lib.cudil_engine_info(self.h, ctypes.byref(m), ctypes.byref(t), ctypes.byref(sb), ctypes.byref(vb))
        return {"mode": m.value, "threads": t.value, "sign_blocks": sb.value, "verify_blocks": vb.value}

    def set_secret_keys(self, d_sk: torch.Tensor, stream=None):
        n = d_sk.numel() // self.params.sk_bytes
        check(lib.cudil_engine_set_secret_keys(self.h, d_sk.data_ptr(), n, _sp(stream)), "set_secret_keys")

    def update_secret_keys(self, d_sk: torch.Tensor, first: int, stream=None):
        """Cache rows first .. first + n - 1 from the n packed secret keys in d_sk (first must not
        exceed the rows built so far); see cudil_engine_update_secret_keys."""
        n = d_sk.numel() // self.params.sk_bytes
        check(lib.cudil_engine_update_secret_keys(self.h, d_sk.data_ptr(), first, n, _sp(stream)),
              "update_secret_keys")

    def attach_keys(self, src: "Engine"):
        """Share src's key caches (same parameter set); src must outlive this engine."""
        check(lib.cudil_engine_attach_keys(self.h, src.h), "attach_keys")
        self._cache_owner = src

    def set_public_keys(self, d_pk: torch.Tensor, stream=None):
        n = d_pk.numel() // self.params.pk_bytes
        check(lib.cudil_engine_set_public_keys(self.h, d_pk.data_ptr(), n, _sp(stream)), "set_public_keys")

    def sign(self, d_sig: torch.Tensor, d_msgs: torch.Tensor, offsets, mlens, key_idx, stream=None,
             d_rhoprime: torch.Tensor | None = None, rho_seed: bytes | None = None, rho_counter: int = 0):
        """d_rhoprime: optional device tensor of 64 random bytes per item (randomized signing);
        rho_seed: optional 32-byte seed from which the device derives every item's rho' as
        SHAKE256(rho_seed || le64(rho_counter + i), 64) (seeded randomized signing)."""
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        mlens = np.ascontiguousarray(mlens, dtype=np.uint32)
        key_idx = np.ascontiguousarray(key_idx, dtype=np.uint32)
        n = len(mlens)
        if rho_seed is not None:
            seed = bytes(rho_seed)
            if len(seed) != 32:
                raise ValueError("rho_seed must be 32 bytes")
            check(lib.cudil_engine_sign_seeded(self.h, d_sig.data_ptr(), d_msgs.data_ptr(), d_msgs.numel(),
                                               offsets.ctypes.data, mlens.ctypes.data, key_idx.ctypes.data, seed,
                                               rho_counter, n, _sp(stream)), "cudil_engine_sign_seeded")
            return
        if d_rhoprime is not None:
            check(lib.cudil_engine_sign_randomized(self.h, d_sig.data_ptr(), d_msgs.data_ptr(), d_msgs.numel(),
                                                   offsets.ctypes.data, mlens.ctypes.data, key_idx.ctypes.data,
                                                   d_rhoprime.data_ptr(), n, _sp(stream)), "cudil_engine_sign_randomized")
            return
        check(lib.cudil_engine_sign(self.h, d_sig.data_ptr(), d_msgs.data_ptr(), d_msgs.numel(), offsets.ctypes.data,
                                    mlens.ctypes.data, key_idx.ctypes.data, n, _sp(stream)), "cudil_engine_sign")

    def verify(self, d_ret: torch.Tensor, d_sig: torch.Tensor, d_msgs: torch.Tensor, offsets, mlens, key_idx,
               stream=None):
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        mlens = np.ascontiguousarray(mlens, dtype=np.uint32)
        key_idx = np.ascontiguousarray(key_idx, dtype=np.uint32)
        n = len(mlens)
        check(lib.cudil_engine_verify(self.h, d_ret.data_ptr(), d_sig.data_ptr(), d_msgs.data_ptr(), d_msgs.numel(),
                                      offsets.ctypes.data, mlens.ctypes.data, key_idx.ctypes.data, n, _sp(stream)),
              "cudil_engine_verify")

    def last_status(self) -> tuple[int, int]:
        a, e = ctypes.c_ulonglong(), ctypes.c_uint32()
        rc = lib.cudil_engine_last_status(self.h, ctypes.byref(a), ctypes.byref(e))
        check(rc, "engine batch")
        return a.value, e.value

    def set_limits(self, nonce_limit: int = 65536, lock_spins: int = 1 << 22, idle_polls: int = 1 << 21):
        """Bounds of the signer's device-side loops (defaults restore the library's); see
        cudil_engine_set_limits."""
        check(lib.cudil_engine_set_limits(self.h, nonce_limit, lock_spins, idle_polls), "set_limits")

    def last_nonces(self, n: int, stream=None) -> np.ndarray:
        """Winning nonce of each of the first n items of the last signing batch (0xFFFFFFFE: the
        item's nonces ran out); deterministic signing ran nonce + 1 attempts for the item."""
        out = np.zeros(max(n, 1), np.uint32)
        check(lib.cudil_engine_last_nonces(self.h, out.ctypes.data, n, _sp(stream)), "last_nonces")
        return out[:n]

    def last_work(self) -> tuple[int, int]:
        """(attempts, inverse NTTs of the rejection checks) of the last signing batch."""
        a, i = ctypes.c_ulonglong(), ctypes.c_ulonglong()
        lib.cudil_engine_last_work(self.h, ctypes.byref(a), ctypes.byref(i))
        return a.value, i.value

    def last_phases(self) -> dict:
        """Signer phase profile of the last batch (block-summed SM cycles and iterations)."""
        cyc = (ctypes.c_ulonglong * 4)()
        it = ctypes.c_uint32()
        lib.cudil_engine_last_phases(self.h, cyc, ctypes.byref(it))
        return {"claim": cyc[0], "keccak": cyc[1], "ntt": cyc[2], "total": cyc[3], "iterations": it.value}

    # ---- numpy conveniences (synchronous)
    def sign_np(self, msgs, key_idx, rhoprime: np.ndarray | None = None) -> np.ndarray:
        d_msgs, offs, lens = pack_messages(msgs)
        n = len(lens)
        d_sig = torch.empty(max(n, 1) * self.params.sig_bytes, dtype=torch.uint8, device="cuda")
        d_rp = None
        if rhoprime is not None:
            d_rp = torch.from_numpy(np.ascontiguousarray(rhoprime, dtype=np.uint8).reshape(-1)).cuda()
        self.sign(d_sig, d_msgs, offs, lens, key_idx, d_rhoprime=d_rp)
        torch.cuda.synchronize()
        self.last_status()
        return d_sig.cpu().numpy()[: n * self.params.sig_bytes].reshape(n, self.params.sig_bytes)

    def verify_np(self, sig: np.ndarray, msgs, key_idx) -> np.ndarray:
        d_msgs, offs, lens = pack_messages(msgs)
        n = len(lens)
        d_sig = torch.from_numpy(np.ascontiguousarray(sig, dtype=np.uint8).reshape(-1)).cuda()
        d_ret = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
        self.verify(d_ret, d_sig, d_msgs, offs, lens, key_idx)
        torch.cuda.synchronize()
        return d_ret.cpu().numpy()[:n]


class EnginePipeline:
    """Runs a stream of batches over ``depth`` engines, each on its own CUDA stream, batch k on
    engine k mod depth (signing or verification).

    The persistent kernels' blocks finish apart: over the last part of a launch more and more SMs
    have no block left.  With one engine on one stream the next batch's key-cache build and prehash
    wait for the whole launch; with an engine per stream they start on the SMs freed at its end,
    and so do the first blocks of the next kernel.  Batches are independent (each engine keeps its
    own caches, queue and scratch), so every batch's results are the same as run alone.  The same
    works from C with one ``cudil_engine`` per stream.

    ``sign`` / ``verify`` return the stream on which the batch completes; the caller keeps a
    batch's input and output buffers alive and unchanged until then (``join`` makes a stream wait
    for every batch).
    """

    def __init__(self, mode: int, max_keys: int, max_items: int, depth: int = 2, threads: int = 0, spec_slots: int = 0,
                 share_keys: bool = False):
        """share_keys: the engines after the first read the first engine's key caches (for resident
        keys: build them once through ``engines[0]``, then sign or verify without d_sk / d_pk).  The
        shared rows are read by batches on every stream, so rebuild them through ``engines[0]``
        only after ``join`` on the stream that builds them."""
        if depth < 1:
            raise ValueError("depth must be at least 1")
        self.engines = [Engine(mode, max_keys, max_items, threads=threads, spec_slots=spec_slots) for _ in range(depth)]
        self.share_keys = share_keys
        if share_keys:
            for e in self.engines[1:]:
                e.attach_keys(self.engines[0])
        self.streams = [torch.cuda.Stream() for _ in range(depth)]
        self.k = 0

    def _check_keys_arg(self, d_keys, name: str):
        if d_keys is not None and self.share_keys:
            raise ValueError(f"{name} per batch needs engines with caches of their own (share_keys=False); with "
                             f"shared caches build them once through engines[0]")

    def _next(self, after):
        j = self.k % len(self.engines)
        self.k += 1
        s = self.streams[j]
        if after is None:
            after = torch.cuda.current_stream()
        if isinstance(after, torch.cuda.Event):
            s.wait_event(after)
        elif after is not False:
            s.wait_stream(after)
        return self.engines[j], s

    def sign(self, d_sig: torch.Tensor, d_msgs: torch.Tensor, offsets, mlens, key_idx, d_sk: torch.Tensor | None = None,
             after=None):
        """Signs the next batch.  d_sk: packed secret keys whose cache rows this batch's engine
        builds first (None: the engine's current rows); after: a stream or event the batch waits
        for, where its inputs are ready (default: the current stream; False: no wait)."""
        self._check_keys_arg(d_sk, "d_sk")
        e, s = self._next(after)
        if d_sk is not None:
            e.set_secret_keys(d_sk, stream=s)
        e.sign(d_sig, d_msgs, offsets, mlens, key_idx, stream=s)
        return s

    def verify(self, d_ret: torch.Tensor, d_sig: torch.Tensor, d_msgs: torch.Tensor, offsets, mlens, key_idx,
               d_pk: torch.Tensor | None = None, after=None):
        """Verifies the next batch (d_pk: packed public keys whose cache rows are built first)."""
        self._check_keys_arg(d_pk, "d_pk")
        e, s = self._next(after)
        if d_pk is not None:
            e.set_public_keys(d_pk, stream=s)
        e.verify(d_ret, d_sig, d_msgs, offsets, mlens, key_idx, stream=s)
        return s

    def join(self, stream=None):
        """Makes `stream` (default: the current stream) wait for every batch run so far."""
        stream = stream or torch.cuda.current_stream()
        for s in self.streams:
            stream.wait_stream(s)

    def close(self):
        for e in reversed(self.engines):  # engines sharing the first one's caches go first
            e.close()


def _sp(stream):
    if stream is None:
        return None
    return stream if isinstance(stream, int) else stream.cuda_stream
