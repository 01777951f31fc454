#!/usr/bin/env python3
"""Benchmark of the batched Dilithium path on B200 (one JSON line on rank 0).

Default workload: Dilithium2 batched signing of a batch of 10000 32-byte messages, one key per
message (the reference's bench_dilithium batch, benches/bench_dilithium.cu:277-296), keys from
the reference's seed scheme SHAKE128(le64(2i+1)).  A step = one sign call over the whole batch
followed by one verify call over the produced signatures.

  value         Dilithium2 signatures/s with inputs resident in HBM (device-pointer C-ABI calls)
  e2e           the same through the public host-buffer C ABI (cudil_sign / cudil_verify with
                pinned host buffers; H2D of m, sk and D2H of sig inside the timed region)
  verify_per_s  verifications/s of the same step (device-resident)
  roofline      dominant kernel of the step: algorithmic 32-bit ALU operations per launch over its
                CUDA-event duration, against the measured LOP3/SHF issue peak of this GPU
  cpu_baseline  the CPU oracle (C restatement, OpenMP over all host cores) on a bounded sample

--impl reference runs the CPU implementation of the same path (the oracle; the reference ships no
CPU Dilithium) on the host cores and prints the same metric.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Dilithium2 sign/s (batched, bit-exact) on 1 B200"
UNIT = "signatures/s"
MLEN = 32

# Algorithmic work model (32-bit ALU operations).  One Keccak-f[1600] permutation lowered to
# 3-input LOP3 and funnel shifts: per round theta 20 (parity) + 20 (D) + 50 (apply), rho 48,
# chi 50, iota 2 = 190; 24 rounds.
OPS_PERM = 24 * 190
OPS_NTT_FWD = 1024 * 6          # 1024 butterflies: 3 IMAD + 3 IADD
OPS_NTT_INV = 1024 * 6 + 256 * 4  # + the final multiplication by f
OPS_PW = 5                        # one Montgomery pointwise product


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------- CPU legs
def cpu_sign_rate(mode: int, budget_s: float, nthreads: int = 0) -> tuple[float, str, int]:
    """Oracle signatures/s on all host threads over a bounded sample of the same workload."""
    from oracle import pyoracle as ora
    cores = os.cpu_count() or 1
    n0 = max(16, cores * 4)
    pk, sk = ora.keypair_batch(mode, n0, 0, nthreads)
    m = ora.messages_from_ctr(n0, MLEN)
    t = time.perf_counter()
    ora.sign_batch(mode, m, sk, nthreads=nthreads)
    dt = max(time.perf_counter() - t, 1e-6)
    n = int(min(20000, max(n0, n0 * budget_s / dt)))
    pk, sk = ora.keypair_batch(mode, n, 0, nthreads)
    m = ora.messages_from_ctr(n, MLEN)
    t = time.perf_counter()
    ora.sign_batch(mode, m, sk, nthreads=nthreads)
    dt = time.perf_counter() - t
    return n / dt, f"{n} Dilithium{mode} signatures of {MLEN}-byte messages (keys 0..{n - 1} of the seed scheme)", cores


def run_reference(args) -> dict:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return {}
    from oracle import pyoracle as ora
    cores = os.cpu_count() or 1
    mode = args.mode
    # bounded sample per step
    n = args.ref_sample
    pk, sk = ora.keypair_batch(mode, n)
    m = ora.messages_from_ctr(n, MLEN)
    for _ in range(args.warmup):
        ora.sign_batch(mode, m[: max(1, n // 8)], sk[: max(1, n // 8)])
    t = time.perf_counter()
    for _ in range(args.steps):
        ora.sign_batch(mode, m, sk)
    dt = time.perf_counter() - t
    v = n * args.steps / dt
    return {
        "metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (reference seed scheme)",
        "config": {"workload": f"Dilithium{mode} sign, {MLEN}-byte messages, CPU sample of {n} per step",
                   "batch": n, "mlen": MLEN},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{n} signatures per step, OpenMP over {cores} threads"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ---------------------------------------------------------------------------- GPU leg
def kernel_ops(name: str, launches: int, mode: int, batch: int, nexec_total: int, mlen: int, pm) -> float | None:
    """Algorithmic ALU operations of all launches of one kernel in the instrumented step."""
    K, L, w1 = pm.k, pm.l, pm.k * pm.polyw1_packed
    blocks = lambda nbytes: nbytes // 136 + 1  # SHAKE256 absorb permutations incl. padding
    if name == "k_expand_a":
        return 2 * batch * K * L * 5 * OPS_PERM  # sign setup + verify
    if name == "k_sign_expand_mask":
        return nexec_total * L * 5 * OPS_PERM
    if name == "k_sign_challenge":
        return nexec_total * (blocks(64 + w1) + 1) * OPS_PERM
    if name == "k_sign_compute_w":
        return nexec_total * (L * OPS_NTT_FWD + K * OPS_NTT_INV + K * L * 256 * OPS_PW)
    if name == "k_sign_prehash":
        return batch * (blocks(32 + mlen) + 1) * OPS_PERM
    if name == "k_verify_prepare":
        return batch * (blocks(pm.pk_bytes) + blocks(32 + mlen) + 1) * OPS_PERM
    if name == "k_verify_final":
        return batch * blocks(64 + w1) * OPS_PERM
    if name == "k_verify_w":
        return batch * ((L + 1 + K) * OPS_NTT_FWD + K * OPS_NTT_INV + (K * L + K) * 256 * OPS_PW)
    if name == "k_sign_unpack_ntt":
        return batch * (L + 2 * K) * OPS_NTT_FWD
    return None


def run_gpu(args) -> dict | None:
    import numpy as np
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))

    import cudilithium_b200 as cd
    from cudilithium_b200 import _lib
    from cudilithium_b200.api import TaskLut, alloc_pool, pinned

    lib = _lib.lib
    mode, B, T = args.mode, args.batch, args.threshold
    d = cd.Dilithium(mode)
    pm = d.params
    dev = torch.device("cuda", local)
    st = torch.cuda.current_stream()
    sp_ptr = st.cuda_stream

    # ---- inputs (reference seed scheme; each rank signs its own batch of the same shape)
    t0 = time.perf_counter()
    kp_pool, kpp = alloc_pool(d.keypair_row_bytes(), B)
    d_pk = torch.empty(B * pm.pk_bytes, dtype=torch.uint8, device=dev)
    d_sk = torch.empty(B * pm.sk_bytes, dtype=torch.uint8, device=dev)
    _lib.check(lib.cudil_keypair_dev(mode, d_pk.data_ptr(), d_sk.data_ptr(), None, kp_pool.data_ptr(), kpp, B,
                                     sp_ptr, rank * 2 * B), "keypair")
    torch.cuda.synchronize()
    kg_ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    kg_ev[0].record(st)
    _lib.check(lib.cudil_keypair_dev(mode, d_pk.data_ptr(), d_sk.data_ptr(), None, kp_pool.data_ptr(), kpp, B,
                                     sp_ptr, rank * 2 * B), "keypair")
    kg_ev[1].record(st)
    torch.cuda.synchronize()
    keygen_ms = kg_ev[0].elapsed_time(kg_ev[1])
    del kp_pool
    rng = np.random.default_rng(1234 + rank)
    m_host = rng.integers(0, 256, (B, MLEN), dtype=np.uint8)
    d_m = torch.from_numpy(m_host.reshape(-1)).to(dev)
    d_sig = torch.empty(B * pm.sig_bytes, dtype=torch.uint8, device=dev)
    d_ret = torch.empty(B, dtype=torch.int32, device=dev)
    s_pool, sp = alloc_pool(d.sign_row_bytes(MLEN), B)
    t_pool, tp = alloc_pool(d.sign_temp_row_bytes(), T)
    v_pool, vp = alloc_pool(d.verify_row_bytes(MLEN), B)
    lut = TaskLut(B, T)
    log(f"[bench] rank {rank}: inputs ready in {time.perf_counter() - t0:.1f}s "
        f"(pools {(s_pool.numel() + t_pool.numel() + v_pool.numel()) / 2**20:.0f} MiB)")

    def sign_dev():
        _lib.check(lib.cudil_sign_dev(mode, d_sig.data_ptr(), pm.sig_bytes, d_m.data_ptr(), MLEN, MLEN,
                                      d_sk.data_ptr(), s_pool.data_ptr(), sp, t_pool.data_ptr(), tp,
                                      ctypes_byref(lut.c), T, B, sp_ptr), "sign")

    def verify_dev():
        _lib.check(lib.cudil_verify_dev(mode, d_ret.data_ptr(), d_sig.data_ptr(), pm.sig_bytes, pm.sig_bytes,
                                        d_m.data_ptr(), MLEN, MLEN, d_pk.data_ptr(), v_pool.data_ptr(), vp, B,
                                        sp_ptr), "verify")

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        sign_dev()
        verify_dev()
    barrier()
    # correctness of the timed configuration: every produced signature verifies
    assert int((d_ret != 0).sum().item()) == 0, "warm-up signatures failed to verify"

    # ---- timed region: K steps, device-resident inputs
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    launches0 = lib.cudil_launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    wall0 = time.perf_counter()
    for a, b, c in ev:
        a.record(st)
        sign_dev()
        b.record(st)
        verify_dev()
        c.record(st)
    barrier()
    wall = time.perf_counter() - wall0
    launches = lib.cudil_launch_count() - launches0
    clk = clocks.stop()
    sign_ms = sum(a.elapsed_time(b) for a, b, _ in ev)
    verify_ms = sum(b.elapsed_time(c) for _, b, c in ev)
    step_ms = sum(a.elapsed_time(c) for a, _, c in ev)
    if world > 1:
        t = torch.tensor([sign_ms, verify_ms, step_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        sign_ms, verify_ms, step_ms = t.tolist()
    value = world * B * args.steps / (sign_ms / 1e3)
    verify_rate = world * B * args.steps / (verify_ms / 1e3)
    ok = int((d_ret != 0).sum().item()) == 0

    # ---- e2e through the host-buffer C ABI
    h_m = pinned(B * MLEN)
    h_m.numpy()[:] = m_host.reshape(-1)
    h_sk = pinned(B * pm.sk_bytes)
    h_sk.copy_(d_sk.cpu())
    h_pk = pinned(B * pm.pk_bytes)
    h_pk.copy_(d_pk.cpu())
    h_sig = pinned(B * pm.sig_bytes)
    h_ret = torch.empty(B, dtype=torch.int32, pin_memory=True)
    siglen = __import__("ctypes").c_size_t(0)

    def sign_host():
        _lib.check(lib.cudil_sign(mode, h_sig.data_ptr(), pm.sig_bytes, ctypes_byref(siglen), h_m.data_ptr(), MLEN,
                                  MLEN, h_sk.data_ptr(), s_pool.data_ptr(), sp, t_pool.data_ptr(), tp,
                                  ctypes_byref(lut.c), T, B, sp_ptr), "sign(host)")

    sign_host()
    barrier()
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for a, b in e2e_ev:
        a.record(st)
        sign_host()
        b.record(st)
    barrier()
    e2e_ms = sum(a.elapsed_time(b) for a, b in e2e_ev)
    if world > 1:
        t = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = t.item()
    e2e = world * B * args.steps / (e2e_ms / 1e3)

    # ---- roofline: one instrumented step, per-kernel CUDA events on the launch stream
    peak_ops = measure_alu_peak(lib, dev, sp_ptr)
    lib.cudil_kernel_stats_reset()
    lib.cudil_kernel_timing(1)
    sign_dev()
    verify_dev()
    torch.cuda.synchronize()
    lib.cudil_kernel_timing(0)
    stats = _lib.kernel_stats()
    nexec_total = stats.get("k_sign_expand_mask", (0, 0))[1] * T
    total_ms = sum(v[0] for v in stats.values())
    dom = max(stats.items(), key=lambda kv: kv[1][0])
    name, (ms, n_launch) = dom
    ops = kernel_ops(name, n_launch, mode, B, nexec_total, MLEN, pm)
    achieved = (ops / n_launch) / (ms / n_launch / 1e3) / 1e9 if ops else None
    roofline = {
        "bound": "int32-alu", "kernel": name, "achieved": achieved, "peak": peak_ops / 1e9, "unit": "Gop/s",
        "frac": (achieved / (peak_ops / 1e9)) if achieved else None, "traffic": None,
        "ms_per_launch": ms / n_launch, "launches": n_launch,
        "share_of_step": ms / total_ms if total_ms else None,
        "peak_source": "measured live: k_alu_peak (3 LOP3 : 1 SHF, the Keccak mix)",
        "kernels": {k: {"ms": round(v[0], 4), "launches": v[1]} for k, v in sorted(stats.items(), key=lambda kv: -kv[1][0])},
    }

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": step_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32", "data": "synthetic: keys from the reference seed scheme, uniform random 32-byte messages",
        "config": {"workload": f"Dilithium{mode} batched sign + verify, batch {B} (reference bench batch), "
                               f"{MLEN}-byte messages, one key per message", "batch": B, "mlen": MLEN,
                   "path": "plain stage-by-stage (cudil_sign_dev / cudil_verify_dev)", "exec_threshold": T,
                   "l2": "inputs larger than L2: sign pool rows alone are "
                         f"{s_pool.numel() / 2**20:.0f} MiB per rank", "parallelism": f"replicas x{world}"},
        "verify_per_s": verify_rate, "keygen_per_s": B / (keygen_ms / 1e3), "all_verified": ok,
        "attempts_per_signature": nexec_total / B if B else None,
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": B * (MLEN + pm.sk_bytes),
                "d2h_bytes_per_step": B * pm.sig_bytes},
        "gpu_launches": int(launches), "wall_s_timed": wall, "clocks": clk, "roofline": roofline,
    }
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, sample, cores = cpu_sign_rate(mode, args.cpu_seconds)
        result["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}
    return result if rank == 0 else None


def ctypes_byref(x):
    import ctypes
    return ctypes.byref(x)


def measure_alu_peak(lib, dev, stream_ptr) -> float:
    """32-bit LOP3/SHF operations per second of this GPU (best of 3 launches, CUDA events)."""
    import ctypes

    import torch
    nsm = torch.cuda.get_device_properties(dev).multi_processor_count
    blocks = nsm * 8
    out = torch.empty(blocks * 256, dtype=torch.int32, device=dev)
    ops = ctypes.c_double(0)
    lib.cudil_alu_peak(out.data_ptr(), blocks, 256, stream_ptr, ctypes.byref(ops))
    best = 0.0
    for _ in range(3):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        st = torch.cuda.current_stream()
        a.record(st)
        lib.cudil_alu_peak(out.data_ptr(), blocks, 4096, stream_ptr, ctypes.byref(ops))
        b.record(st)
        torch.cuda.synchronize()
        best = max(best, ops.value / (a.elapsed_time(b) / 1e3))
    return best


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["cudil", "reference"], default="cudil")
    ap.add_argument("--mode", type=int, default=2, choices=[2, 3, 5])
    ap.add_argument("--batch", type=int, default=10000)
    ap.add_argument("--threshold", type=int, default=16384, help="exec slots per rejection round (plain path)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-sample", type=int, default=4000)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        log("[bench] warmup raised to 3 (minimum)")
        args.warmup = 3
    if args.impl == "reference":
        res = run_reference(args)
    else:
        res = run_gpu(args)
    if res:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
