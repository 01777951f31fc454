"""Continuous-batching request server: Python driver of ``cudil_serve_trace`` (include/cudilithium.h).

The server itself is host C++ inside the library (``csrc/server.cu``): one FIFO per (parameter
set, operation) lane, batch slots per lane with their own stream and device buffers, admission of
slots by a device-memory budget, and either fused engines sharing one resident key cache per
parameter set (path 0) or the plain stage-by-stage calls (path 1).  This module builds seeded
open-loop traces, runs them and summarises latency and throughput.

    keys = make_keys({2: 4096, 3: 4096, 5: 4096})
    tr = poisson_trace(keys, rate=1e6, n=200_000, seed=1)
    res = serve(tr, keys, path=0, budget_bytes=8 << 30)
    print(summary(tr, res))
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import check, lib

MODES = (2, 3, 5)
REQUEST_DTYPE = np.dtype([("arrival_s", "<f8"), ("mode", "<i4"), ("op", "<i4"), ("key", "<u4"),
                          ("mlen", "<u4"), ("msg_off", "<u8"), ("sig_off", "<u8")], align=True)
RESULT_DTYPE = np.dtype([("done_s", "<f8"), ("status", "<i4"), ("batch_size", "<u4")], align=True)
SIGN, VERIFY = 0, 1


@dataclass
class Keys:
    """Seeded key pairs per parameter set, host copies (rows of sk_bytes / pk_bytes)."""
    sk: dict = field(default_factory=dict)
    pk: dict = field(default_factory=dict)

    def n(self, mode: int) -> int:
        return 0 if mode not in self.sk else len(self.sk[mode]) // _lib.params(mode).sk_bytes


@dataclass
class Trace:
    reqs: np.ndarray          # REQUEST_DTYPE, arrival order
    msgs: np.ndarray          # uint8, all messages back to back
    sigs: np.ndarray          # uint8, signatures of verify requests (sig_off indexes here)
    expect: np.ndarray        # int32, expected verify status (0 valid / -1 tampered); 0 for sign
    rate: float               # offered requests per second (inf: everything arrives at t = 0)


def make_keys(counts: dict, seed: int = 7) -> Keys:
    """counts[mode] key pairs per parameter set, generated on the GPU from seeded indices
    (reference keypair seeding: SHAKE128(le64(rand_index + 2i + 1)))."""
    from .api import Dilithium
    k = Keys()
    for mode, n in counts.items():
        if n <= 0:
            continue
        d = Dilithium(mode)
        pk, sk = d.keypair(n, rand_index=seed * 1_000_003 + mode)
        k.pk[mode] = np.ascontiguousarray(pk).reshape(-1)
        k.sk[mode] = np.ascontiguousarray(sk).reshape(-1)
    return k


def _log_uniform(rng, lo: int, hi: int, n: int) -> np.ndarray:
    """Integers in [lo, hi] with log-uniform density (lo = 0: log-uniform over [1, hi + 1], minus 1)."""
    s = 1 if lo == 0 else 0
    v = np.floor(np.exp(rng.uniform(np.log(lo + s), np.log(hi + s + 1), n))) - s
    return np.clip(v, lo, hi).astype(np.uint32)


def poisson_trace(keys: Keys, rate: float, n: int, seed: int = 1, mix=(0.60, 0.25, 0.15), verify_frac: float = 0.70,
                  mlen_range=(32, 4096), tamper_frac: float = 0.05, modes=MODES) -> Trace:
    """Open-loop trace: exponential inter-arrival times at `rate` requests/s (rate = inf: all at
    t = 0), parameter set by `mix`, verify with probability `verify_frac`, key uniform over the
    parameter set's keys, message length log-uniform over `mlen_range`, uniform random bytes.
    Verify requests get a signature made by the fused engine; `tamper_frac` of them get one random
    bit flipped (expected status -1)."""
    rng = np.random.default_rng(seed)
    mix = np.asarray([mix[MODES.index(m)] for m in modes], dtype=np.float64)
    mix /= mix.sum()
    reqs = np.zeros(n, dtype=REQUEST_DTYPE)
    if np.isinf(rate):
        reqs["arrival_s"] = 0.0
    else:
        reqs["arrival_s"] = np.cumsum(rng.exponential(1.0 / rate, n))
    reqs["mode"] = np.asarray(modes)[rng.choice(len(modes), n, p=mix)]
    reqs["op"] = (rng.random(n) < verify_frac).astype(np.int32)
    for m in modes:
        sel = reqs["mode"] == m
        reqs["key"][sel] = rng.integers(0, keys.n(m), int(sel.sum()))
    reqs["mlen"] = _log_uniform(rng, mlen_range[0], mlen_range[1], n)
    offs = np.zeros(n, dtype=np.uint64)
    offs[1:] = np.cumsum(reqs["mlen"][:-1].astype(np.uint64))
    reqs["msg_off"] = offs
    msgs = rng.integers(0, 256, int(reqs["mlen"].sum()) + 8, dtype=np.uint8)

    # signatures of the verify requests, by parameter set
    expect = np.zeros(n, dtype=np.int32)
    sig_chunks, pos = [], 0
    for m in modes:
        idx = np.nonzero((reqs["mode"] == m) & (reqs["op"] == VERIFY))[0]
        if len(idx) == 0:
            continue
        sb = _lib.params(m).sig_bytes
        sig = sign_messages(m, keys, [msgs[int(o): int(o) + int(l)] for o, l in zip(reqs["msg_off"][idx], reqs["mlen"][idx])],
                            reqs["key"][idx])
        bad = rng.random(len(idx)) < tamper_frac
        for j in np.nonzero(bad)[0]:
            bit = int(rng.integers(0, sb * 8))
            sig[j, bit // 8] ^= np.uint8(1 << (bit % 8))
        expect[idx[bad]] = -1
        reqs["sig_off"][idx] = pos + np.arange(len(idx), dtype=np.uint64) * sb
        sig_chunks.append(sig.reshape(-1))
        pos += len(idx) * sb
    sigs = np.concatenate(sig_chunks) if sig_chunks else np.zeros(8, np.uint8)
    return Trace(reqs, msgs, sigs, expect, float(rate))


def sign_messages(mode: int, keys: Keys, msgs: list, key_idx: np.ndarray) -> np.ndarray:
    """Deterministic signatures of msgs[i] under key key_idx[i] via the fused engine."""
    from .engine import Engine, pack_messages
    pm = _lib.params(mode)
    n = len(msgs)
    nk = keys.n(mode)
    e = Engine(mode, nk, n)
    try:
        sk = torch.from_numpy(keys.sk[mode]).cuda()
        e.set_secret_keys(sk)
        buf, offs, lens = pack_messages([bytes(m) for m in msgs])
        sig = torch.empty(n * pm.sig_bytes, dtype=torch.uint8, device="cuda")
        e.sign(sig, buf, offs, lens, np.asarray(key_idx, dtype=np.uint32))
        torch.cuda.synchronize()
        e.last_status()
        return sig.cpu().numpy().reshape(n, pm.sig_bytes)
    finally:
        e.close()


def serve(tr: Trace, keys: Keys, path: int = 0, budget_bytes: int = 0, slots_per_lane: int = 2, max_batch: int = 8192,
          threads: int = 0, spec_slots: int = 0, plain_exec_threshold: int = 0, want_sigs: bool = True,
          slots_by_load: bool = True):
    """Replays `tr` through cudil_serve_trace.  slots_by_load: lanes get batch slots in proportion
    to their share of the requests (at least slots_per_lane).  Returns (results[RESULT_DTYPE],
    signatures (n, max sig bytes) or None, stats dict)."""
    from .autotune import tuned
    n = len(tr.reqs)
    cfg = _lib.cudil_serve_config()
    cfg.device_budget_bytes = budget_bytes
    cfg.path = path
    cfg.slots_per_lane = slots_per_lane
    cfg.max_batch = max_batch
    t = tuned(2)
    cfg.engine_threads = threads or t["threads"]
    cfg.engine_spec_slots = spec_slots or t["spec_slots"]
    cfg.plain_exec_threshold = plain_exec_threshold or max(1024, max_batch)
    cfg.max_mlen = max(1, int(tr.reqs["mlen"].max()) if n else 1)
    cfg.lane_slots_by_load = 1 if slots_by_load else 0
    sk = (ctypes.c_void_p * 3)()
    pk = (ctypes.c_void_p * 3)()
    nk = (ctypes.c_size_t * 3)()
    keep = []
    for i, m in enumerate(MODES):
        if m in keys.sk:
            a, b = np.ascontiguousarray(keys.sk[m]), np.ascontiguousarray(keys.pk[m])
            keep += [a, b]
            sk[i], pk[i], nk[i] = a.ctypes.data, b.ctypes.data, keys.n(m)
    reqs = np.ascontiguousarray(tr.reqs)
    res = np.zeros(n, dtype=RESULT_DTYPE)
    sig_pitch = max(_lib.params(m).sig_bytes for m in MODES)
    sig_out = np.zeros((n, sig_pitch), dtype=np.uint8) if want_sigs else None
    st = _lib.cudil_serve_stats()
    rc = lib.cudil_serve_trace(ctypes.byref(cfg), sk, pk, nk, reqs.ctypes.data, n, tr.msgs.ctypes.data,
                               tr.sigs.ctypes.data, sig_out.ctypes.data if want_sigs else None, sig_pitch,
                               res.ctypes.data, ctypes.byref(st))
    check(rc, "cudil_serve_trace")
    return res, sig_out, {"wall_s": st.wall_s, "batches": st.batches, "slots": st.slots,
                          "device_bytes": st.device_bytes, "host_stage_s": st.host_stage_s,
                          "device_wait_s": st.device_wait_s, "host_post_s": st.host_post_s}


def summary(tr: Trace, res: np.ndarray, stats: dict) -> dict:
    """Throughput (requests completed / wall time) and latency percentiles in ms, overall and per
    lane."""
    lat = (res["done_s"] - tr.reqs["arrival_s"]) * 1e3
    out = {"requests": int(len(res)), "offered_per_s": tr.rate, "wall_s": stats["wall_s"],
           "throughput_per_s": len(res) / stats["wall_s"] if stats["wall_s"] > 0 else 0.0,
           "p50_ms": float(np.percentile(lat, 50)) if len(lat) else 0.0,
           "p99_ms": float(np.percentile(lat, 99)) if len(lat) else 0.0,
           "mean_batch": float(res["batch_size"].mean()) if len(res) else 0.0,
           "batches": stats["batches"], "slots": stats["slots"], "device_bytes": stats["device_bytes"],
           "slot_time_s": {k: stats[k] for k in ("host_stage_s", "device_wait_s", "host_post_s")}, "lanes": {}}
    for m in MODES:
        for op, name in ((SIGN, "sign"), (VERIFY, "verify")):
            sel = (tr.reqs["mode"] == m) & (tr.reqs["op"] == op)
            if sel.any():
                out["lanes"][f"d{m}_{name}"] = {"n": int(sel.sum()), "p50_ms": float(np.percentile(lat[sel], 50)),
                                                 "p99_ms": float(np.percentile(lat[sel], 99))}
    return out
