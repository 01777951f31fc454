"""Autotuner for the fused engine: picks the signer kernel (phased or asynchronous), the block
size and the per-block speculation target for each parameter set by timing real signing batches
(a stream of batches over two engines, as EnginePipeline runs them), and caches the result as JSON
(``cudilithium_b200/tuned.json``, keyed by GPU name).

    python -m cudilithium_b200.autotune [--modes 2 3 5] [--batch 16384]

``Engine(..., threads=0)`` and ``tuned(mode)`` read the cache; without an entry for this GPU
the built-in defaults below apply.
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

TUNED_PATH = Path(__file__).resolve().parent / "tuned.json"
# measured on B200 (Dilithium2, 10000 and 65536 single-use keys): 256 threads per block and a
# per-block target of 32 attempts in flight gave the highest signing throughput
DEFAULTS = {2: {"threads": 256, "spec_slots": 32, "sign_kernel": 0},
            3: {"threads": 256, "spec_slots": 32, "sign_kernel": 0},
            5: {"threads": 256, "spec_slots": 32, "sign_kernel": 0}}
THREADS = (128, 256)
SPEC = (16, 32, 64, 128)
# asynchronous signer variants (kernel, speculation target = its slot count).  The phased kernel
# with one wide block per SM (variant 5) is left out: it wins on isolated batches of 10 000 and
# more, but serves small batches (the serving loop's) and the end-to-end step with host-memory
# output worse than the 256-thread phased kernel; callers with large batches select it explicitly.
ASYNC = ((2, 128), (3, 160))
ROUNDS = 3
PIPE_BATCHES = 6


def _gpu_name() -> str:
    import torch
    return torch.cuda.get_device_name(torch.cuda.current_device()) if torch.cuda.is_available() else "cpu"


def tuned(mode: int) -> dict:
    """Tuned engine settings for this GPU (falls back to DEFAULTS)."""
    try:
        data = json.loads(TUNED_PATH.read_text())
        return data.get(_gpu_name(), {}).get(str(mode), DEFAULTS[mode])
    except (OSError, ValueError):
        return DEFAULTS[mode]


def tune_mode(mode: int, batch: int) -> dict:
    import numpy as np
    import torch

    import cudilithium_b200 as cd
    from cudilithium_b200.api import alloc_pool
    from cudilithium_b200.engine import Engine
    lib = cd.lib
    d = cd.Dilithium(mode)
    pm = d.params
    dev = torch.device("cuda")
    spp = torch.cuda.current_stream().cuda_stream
    pool, kpp = alloc_pool(d.keypair_row_bytes(), batch)
    pk = torch.empty(batch * pm.pk_bytes, dtype=torch.uint8, device=dev)
    sk = torch.empty(batch * pm.sk_bytes, dtype=torch.uint8, device=dev)
    lib.cudil_keypair_dev(mode, pk.data_ptr(), sk.data_ptr(), None, pool.data_ptr(), kpp, batch, spp, 0)
    del pool
    m = torch.randint(0, 256, (batch * 32,), dtype=torch.uint8, device=dev)
    offs = np.arange(batch, dtype=np.uint64) * 32
    lens = np.full(batch, 32, np.uint32)
    keys = np.arange(batch, dtype=np.uint32)
    sig = torch.empty(batch * pm.sig_bytes, dtype=torch.uint8, device=dev)
    # Every candidate signs a stream of PIPE_BATCHES batches over two engines on two streams (the
    # way EnginePipeline runs batches: the next batch starts on the SMs the current signer frees),
    # and is timed in ROUNDS interleaved rounds (its median is kept), so that a slow moment of the
    # GPU does not decide between two settings within a few per cent of each other.
    engines = {}
    cands = []
    for t in THREADS:
        pair = [Engine(mode, batch, batch, threads=t) for _ in range(2)]
        for e in pair:
            e.set_secret_keys(sk, stream=spp)
        engines[t] = pair
        cands += [(t, 0, s) for s in SPEC] + ([(t, v, s) for v, s in ASYNC] if t == THREADS[-1] else [])
    streams = [torch.cuda.Stream() for _ in range(2)]
    sigs = [torch.empty_like(sig) for _ in range(2)]
    times = {c: [] for c in cands}
    ref = None
    for _ in range(ROUNDS):
        for t, kern, s in cands:
            pair = engines[t]
            for e in pair:
                e.set_sign_kernel(kern)
                e.set_spec_slots(s)
            pair[0].sign(sig, m, offs, lens, keys, stream=spp)
            torch.cuda.synchronize()
            if ref is None:
                ref = sig.clone()
            assert torch.equal(sig, ref), "tuning candidates disagree"
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for x in streams:
                x.wait_event(a)
            for k in range(PIPE_BATCHES):
                pair[k % 2].sign(sigs[k % 2], m, offs, lens, keys, stream=streams[k % 2])
            cur = torch.cuda.current_stream()
            for x in streams:
                cur.wait_stream(x)
            b.record()
            torch.cuda.synchronize()
            times[(t, kern, s)].append(a.elapsed_time(b) / PIPE_BATCHES)
    for pair in engines.values():
        for e in pair:
            e.close()
    results = []
    for (t, kern, s), ts in times.items():
        ms = sorted(ts)[len(ts) // 2]
        results.append({"threads": t, "spec_slots": s, "sign_kernel": kern, "ms": ms, "sign_per_s": batch / (ms / 1e3)})
    best = min(results, key=lambda r: r["ms"])
    return {"threads": best["threads"], "spec_slots": best["spec_slots"], "sign_kernel": best["sign_kernel"], "batch": batch,
            "sign_per_s": best["sign_per_s"], "candidates": results, "when": time.strftime("%Y-%m-%dT%H:%M:%S")}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--modes", type=int, nargs="+", default=[2, 3, 5])
    ap.add_argument("--batch", type=int, default=16384)
    args = ap.parse_args()
    name = _gpu_name()
    data = {}
    if TUNED_PATH.exists():
        try:
            data = json.loads(TUNED_PATH.read_text())
        except ValueError:
            data = {}
    entry = data.setdefault(name, {})
    for mode in args.modes:
        r = tune_mode(mode, args.batch)
        entry[str(mode)] = r
        print(json.dumps({"mode": mode, "threads": r["threads"], "spec_slots": r["spec_slots"], "sign_kernel": r["sign_kernel"],
                          "sign_per_s": round(r["sign_per_s"])}), flush=True)
    TUNED_PATH.write_text(json.dumps(data, indent=1))


if __name__ == "__main__":
    main()
