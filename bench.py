#!/usr/bin/env python
"""Benchmark of the FSS hot path on B200: DCF evaluation at n = 32 over Z_2^32.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (one step): one party's DCF evaluation of 2^24 elements with input width n = 32,
output ring Z_2^32 (uint32), groupSize 1, keys in the reference byte layout (652 B/element)
— the plain drop-in DCF configuration. Inputs are seeded synthetic: alpha, beta, x uniform,
128-bit seeds uniform, maskedX = x + alpha. Keys are generated on the device before timing
(they are preprocessed material). The 10.9 GB of keys and the 268 MB of seeds exceed the
126 MB L2, so no flush is needed between steps.

`value` is device-timed throughput (CUDA events on the launch stream, inputs resident);
`e2e` is the same through the public API with the per-step maskedX copied in from pinned
host memory and the shares copied back (keys and seeds stay device-resident, as in a
two-party deployment). With torchrun, every rank evaluates its own 2^24 elements (weak
scaling, no data-path collective); times are the max over ranks.

`--impl reference` times the reference's own CPU implementation (FastFss_cpu_dcfEval built
from its sources into oracle/_ref) on a bounded sample with all host threads.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_BITS = 32
ES = 4
N_ELEMENTS = 1 << 24
KEY_BYTES_PER_ELEM = 16 * N_BITS + ES * N_BITS + 2 * ES + ES  # 652
ALGO_BYTES_PER_ELEM = KEY_BYTES_PER_ELEM + 16 + ES + ES  # key + seed + maskedX + share = 676
# Evaluation work per element, in shared-memory table lookups. Per level: one key schedule
# (40 S-box lookups), the seed block of the child on the input's path (160) and its value
# block (160), less the 14 first-round lookups the two blocks share (their plaintexts differ
# only in bytes 0 and 8) and the 12 last-round lookups of value bytes a 32-bit output never
# reads: 40 + 160 + 134 = 334.
LOOKUPS_PER_ELEM = N_BITS * (40 + 160 + 134)
AES_BLOCKS_PER_ELEM = 2 * N_BITS
AES_KS_PER_ELEM = N_BITS
METRIC = "DCF eval Gelem/s at n=32 (Z_2^32), plain vs batched; serving p50/p99 ms"
UNIT = "Gelem/s"
CONFIG = {"workload": "plain DCF eval, 2^24 elements, n=32, Z_2^32 (uint32), groupSize 1, one party per step",
          "elements_per_rank": N_ELEMENTS, "bitWidthIn": N_BITS, "bitWidthOut": N_BITS, "elementSize": ES,
          "groupSize": 1, "key_layout": "reference (sCW region + per-element vCW/tCW/lastCW)",
          "l2": "inputs larger than L2 (10.9 GB keys), no flush"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--elements", type=int, default=N_ELEMENTS)
    ap.add_argument("--cpu-seconds", type=float, default=4.0, help="wall budget of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the DPF, Grotto, batched and serving measurements")
    ap.add_argument("--sections", default="dpf,grotto,batched,serving",
                    help="comma-separated extra measurements to run after the DCF line")
    ap.add_argument("--dpf-all-keys", type=int, default=1 << 12, help="keys of the full-domain DPF measurement")
    ap.add_argument("--batched-instances", type=int, default=256)
    ap.add_argument("--serving-requests", type=int, default=160)
    return ap.parse_args()


# ------------------------------------------------------------------------------------------
# clocks
# ------------------------------------------------------------------------------------------

class ClockSampler:
    """Samples nvidia-smi during the timed region (SM clock, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self, t0: float | None = None, t1: float | None = None) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = [ln for ts, ln in self.lines if t0 is None or (t0 - 0.25 <= ts <= t1 + 0.25)]
        if not lines:
            lines = [ln for _, ln in self.lines]
        for ln in lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------------------------------
# CPU reference timing
# ------------------------------------------------------------------------------------------

def cpu_reference_rate(seconds: float, sample: int = 1 << 18) -> dict:
    """Times the reference's FastFss_cpu_dcfEval (oracle/_ref) — or, if that library is not
    built, the oracle restatement — on a `sample`-element batch of the same workload, with all
    host threads, repeating for about `seconds` of wall time."""
    from oracle.pyoracle import Oracle, RefCpu

    threads = os.cpu_count() or 1
    if RefCpu.available():
        impl, kind = RefCpu(), "reference"
    else:
        impl, kind = Oracle(), "port"
    impl.set_threads(threads)
    rng = np.random.default_rng(1)
    a = rng.integers(0, 2**32, size=sample, dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, 2**32, size=sample, dtype=np.uint64).astype(np.uint32)
    s0 = rng.integers(0, 256, size=sample * 16, dtype=np.uint8)
    s1 = rng.integers(0, 256, size=sample * 16, dtype=np.uint8)
    x = rng.integers(0, 2**32, size=sample, dtype=np.uint64).astype(np.uint32)
    key = impl.dcf_keygen(a, b, s0, s1, N_BITS, N_BITS, 1)
    impl.dcf_eval(x, key, s0, 0, N_BITS, N_BITS, 1)  # warm-up
    reps, t0 = 0, time.perf_counter()
    while True:
        impl.dcf_eval(x, key, s0, 0, N_BITS, N_BITS, 1)
        reps += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    rate = sample * reps / el
    return {"value": rate / 1e9, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"{reps} x FastFss_cpu_dcfEval over {sample} elements (n=32, u32, one party), {el:.2f} s wall"}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.pyoracle import Oracle, RefCpu

    threads = os.cpu_count() or 1
    if RefCpu.available():
        impl, kind = RefCpu(), "reference"
    else:
        impl, kind = Oracle(), "port"
    impl.set_threads(threads)
    sample = 1 << 17
    rng = np.random.default_rng(2)
    a = rng.integers(0, 2**32, size=sample, dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, 2**32, size=sample, dtype=np.uint64).astype(np.uint32)
    s0 = rng.integers(0, 256, size=sample * 16, dtype=np.uint8)
    s1 = rng.integers(0, 256, size=sample * 16, dtype=np.uint8)
    x = rng.integers(0, 2**32, size=sample, dtype=np.uint64).astype(np.uint32)
    key = impl.dcf_keygen(a, b, s0, s1, N_BITS, N_BITS, 1)
    for _ in range(args.warmup):
        impl.dcf_eval(x, key, s0, 0, N_BITS, N_BITS, 1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        impl.dcf_eval(x, key, s0, 0, N_BITS, N_BITS, 1)
    el = time.perf_counter() - t0
    value = sample * args.steps / el / 1e9
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": dict(CONFIG, reference_sample_elements=sample),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": f"each step = FastFss_cpu_dcfEval over {sample} of the 2^24 elements"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------
# GPU run
# ------------------------------------------------------------------------------------------

def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist

    import fastfunctionsecretsharing_b200 as F
    from fastfunctionsecretsharing_b200 import _lib
    from fastfunctionsecretsharing_b200.sharding import max_over_ranks

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    N = args.elements
    gen = torch.Generator(device=dev).manual_seed(1234 + rank)
    alpha = torch.randint(-2**31, 2**31, (N,), dtype=torch.int32, device=dev, generator=gen)
    beta = torch.randint(-2**31, 2**31, (N,), dtype=torch.int32, device=dev, generator=gen)
    seed0 = torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device=dev, generator=gen)
    seed1 = torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device=dev, generator=gen)
    x = torch.randint(-2**31, 2**31, (N,), dtype=torch.int32, device=dev, generator=gen)
    masked = x + alpha
    key = torch.empty(0, dtype=torch.uint8, device=dev)
    F.dcf_key_gen(key, alpha, beta, seed0, seed1, N_BITS, N_BITS, 1)
    # key generation (the dealer's side, not part of the timed step): a second, timed run
    kg0, kg1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    kg0.record()
    F.dcf_key_gen(key, alpha, beta, seed0, seed1, N_BITS, N_BITS, 1)
    kg1.record()
    torch.cuda.synchronize(dev)
    keygen_ms = kg0.elapsed_time(kg1)
    del seed1, x
    out = torch.empty(0, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)

    torch.cuda.synchronize(dev)

    def step():
        F.dcf_eval(out, masked, key, seed0, 0, N_BITS, N_BITS, 1)

    # nvidia-smi starts before the warm-up so its start-up never lands in the timed region
    clocks = ClockSampler(local).__enter__()
    time.sleep(1.0)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    barrier()
    torch.cuda.synchronize(dev)

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    t_begin = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    wall0 = time.time()
    t_begin.record(stream)
    for i in range(args.steps):
        starts[i].record(stream)
        step()
        ends[i].record(stream)
    t_end.record(stream)
    torch.cuda.synchronize(dev)
    wall1 = time.time()
    barrier()
    torch.cuda.synchronize(dev)
    total_ms = t_begin.elapsed_time(t_end)
    kernel_ms = statistics.mean(s.elapsed_time(e) for s, e in zip(starts, ends))
    total_ms = max_over_ranks(total_ms, world)
    kernel_ms = max_over_ranks(kernel_ms, world)
    ms_per_step = total_ms / args.steps
    value = N * world * args.steps / (total_ms / 1e3) / 1e9

    # ---- end to end through the public API, host buffers, H2D + D2H per step ----
    # Every step copies its maskedX in from pinned host memory and its shares back out. Two
    # device buffers and separate H2D and D2H copy streams (ordered by events) let step i + 1's
    # input copy and step i - 1's output copy run while step i is evaluated.
    host_x = masked.cpu().pin_memory()
    host_out = [torch.empty(N, dtype=torch.int32).pin_memory() for _ in range(2)]
    dev_x = [torch.empty_like(masked) for _ in range(2)]
    dev_out = [torch.empty(0, dtype=torch.int32, device=dev) for _ in range(2)]
    h2d_stream = torch.cuda.Stream(dev)
    copy_stream = torch.cuda.Stream(dev)  # device -> host
    h2d_done = [torch.cuda.Event() for _ in range(2)]
    comp_done = [torch.cuda.Event() for _ in range(2)]
    d2h_done = [torch.cuda.Event() for _ in range(2)]

    def e2e_steps(k):
        for i in range(k):
            b = i % 2
            with torch.cuda.stream(h2d_stream):
                if i >= 2:
                    h2d_stream.wait_event(comp_done[b])  # dev_x[b] was read by step i - 2
                dev_x[b].copy_(host_x, non_blocking=True)
                h2d_done[b].record(h2d_stream)
            stream.wait_event(h2d_done[b])
            if i >= 2:
                stream.wait_event(d2h_done[b])  # dev_out[b] was copied out by step i - 2
            F.dcf_eval(dev_out[b], dev_x[b], key, seed0, 0, N_BITS, N_BITS, 1)
            comp_done[b].record(stream)
            with torch.cuda.stream(copy_stream):
                copy_stream.wait_event(comp_done[b])
                host_out[b].copy_(dev_out[b].view(-1), non_blocking=True)
                d2h_done[b].record(copy_stream)

    e2e_steps(args.warmup)
    torch.cuda.synchronize(dev)
    barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(h2d_stream)
    stream.wait_event(e0)
    copy_stream.wait_event(e0)
    e2e_steps(args.steps)
    copy_stream.wait_stream(stream)
    copy_stream.wait_stream(h2d_stream)
    e1.record(copy_stream)
    torch.cuda.synchronize(dev)
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world)
    e2e_value = N * world * args.steps / (e2e_ms / 1e3) / 1e9
    e2e_ok = bool(torch.equal(host_out[(args.steps - 1) % 2], out.view(-1).cpu()))
    clocks.__exit__(None, None, None)

    # ---- correctness of what was timed: party-1 shares reconstruct beta * [maskedX < alpha] ----
    y1 = torch.empty(0, dtype=torch.int32, device=dev)
    F.dcf_eval(out, masked, key, seed0, 0, N_BITS, N_BITS, 1)
    F.dcf_eval(y1, masked, key, seed1_regen(gen_seed=1234 + rank, N=N, dev=dev), 1, N_BITS, N_BITS, 1)
    lt = (masked.to(torch.int64) & 0xFFFFFFFF) < (alpha.to(torch.int64) & 0xFFFFFFFF)
    ok = bool(torch.equal((out + y1).view(-1), torch.where(lt, beta, torch.zeros_like(beta))))

    # ---- roofline: measured shared-memory lookup peak ----
    sink = torch.empty(4 * 512 * 1024, dtype=torch.uint8, device=dev)
    lk = ctypes.c_ulonglong(0)
    h = ctypes.c_void_p(stream.cuda_stream)
    probe = _lib.fn("FastFss_b200_smemLookupProbe")
    iters = 20000
    for _ in range(2):
        probe(sink.data_ptr(), sink.numel(), iters, ctypes.byref(lk), ctypes.byref(h))
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    for _ in range(5):
        probe(sink.data_ptr(), sink.numel(), iters, ctypes.byref(lk), ctypes.byref(h))
    p1.record(stream)
    torch.cuda.synchronize(dev)
    peak_glookups = lk.value * 5 / (p0.elapsed_time(p1) / 1e3) / 1e9

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return

    achieved_glookups = LOOKUPS_PER_ELEM * N / (kernel_ms / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "dcf_eval_n32_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get("dram_bytes_per_launch")
    peaks = {}
    ppath = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(ppath):
        with open(ppath) as f:
            peaks = json.load(f)
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    hbm_ach = ALGO_BYTES_PER_ELEM * N / (kernel_ms / 1e3) / 1e9
    ck = clocks.summary(wall0, wall1)
    nominal = None
    if ck.get("sm_mhz"):
        nominal = FastFssSm(_lib) * 32 * ck["sm_mhz"] * 1e6 / 1e9

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded uniform alpha, beta, x, 128-bit seeds)", "config": CONFIG,
        "roofline": {"bound": "smem", "achieved": achieved_glookups, "peak": peak_glookups, "unit": "Glookup/s",
                     "frac": achieved_glookups / peak_glookups, "traffic": traffic,
                     "peak_source": "measured on this GPU by FastFss_b200_smemLookupProbe (conflict-free LDS)",
                     "nominal_peak_at_sampled_clock": nominal,
                     "algorithmic_lookups_per_element": LOOKUPS_PER_ELEM,
                     "hbm": {"achieved": hbm_ach, "peak": hbm_peak, "unit": "GB/s", "frac": hbm_ach / hbm_peak,
                             "algorithmic_bytes_per_element": ALGO_BYTES_PER_ELEM,
                             "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback"}},
        "kernel_ms": kernel_ms,
        "aes_blocks_per_s": AES_BLOCKS_PER_ELEM * N * world / (kernel_ms / 1e3),
        "aes_key_expansions_per_s": AES_KS_PER_ELEM * N * world / (kernel_ms / 1e3),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": N * ES, "d2h_bytes_per_step": N * ES,
                "shares_match_device_run": e2e_ok,
                "note": ("public API (fastfunctionsecretsharing_b200.dcf_eval -> FastFss_cuda_dcfEval); each step copies "
                         "maskedX in from pinned host memory and the shares out; a step's input and output copies "
                         "overlap the neighbouring steps' evaluations (two buffers, separate H2D and D2H streams); "
                         "keys/seeds stay device-resident")},
        "gpu_launches": args.steps,
        "gpu_launches_e2e": args.steps,
        "clocks": ck,
        "shares_reconstruct": ok,
        "keygen": {"ms": keygen_ms, "Gkeys_per_s": N / (keygen_ms / 1e3) / 1e9,
                   "note": "FastFss_cuda_dcfKeyGen of the same 2^24 keys (both parties' trees per element)"},
    }
    if not args.no_extras:
        del key, seed0
        torch.cuda.empty_cache()
        sections = set(args.sections.split(","))
        if "dpf" in sections:
            line["dpf"] = dpf_section(dev, args, peak_glookups)
        if "grotto" in sections:
            line["grotto_full_domain"] = grotto_section(dev, args, peak_glookups)
        if "batched" in sections:
            line["batched"] = batched_section(dev, args, peak_glookups)
        if "serving" in sections:
            line["serving"] = serving_section(dev, args)
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_reference_rate(args.cpu_seconds)
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def _timed(fn, dev, steps, warmup=3):
    """Mean device ms of fn over `steps` calls on the current stream, after `warmup` calls."""
    import torch

    stream = torch.cuda.current_stream(dev)
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    return e0.elapsed_time(e1) / steps


# DPF evaluation per element at n = 32, groupSize 1, 32-bit output: per level one key schedule
# (40 lookups) and the path child's block (160); the leaf convert is one key schedule and one
# block of which a 32-bit output reads 4 of the 16 last-round bytes (40 + 148).
DPF_LOOKUPS_PER_ELEM = N_BITS * 200 + 40 + 148


def dpf_section(dev, args, peak_glookups) -> dict:
    """Plain DPF eval, 2^24 elements, n = 32 over Z_2^32 (uint32), groupSize 1, one party per
    step; keys 16 B x 32 sCW + tCW + lastCW per element, larger than L2."""
    import torch

    import fastfunctionsecretsharing_b200 as F

    N = args.elements
    gen = torch.Generator(device=dev).manual_seed(4321)
    alpha = torch.randint(-2**31, 2**31, (N,), dtype=torch.int32, device=dev, generator=gen)
    beta = torch.randint(-2**31, 2**31, (N,), dtype=torch.int32, device=dev, generator=gen)
    s0 = torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device=dev, generator=gen)
    s1 = torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device=dev, generator=gen)
    x = torch.randint(-2**31, 2**31, (N,), dtype=torch.int32, device=dev, generator=gen)
    x[: N // 16] = 0  # a sixteenth of the points hit alpha
    masked = x + alpha
    key = torch.empty(0, dtype=torch.uint8, device=dev)
    F.dpf_key_gen(key, alpha, beta, s0, s1, N_BITS, N_BITS, 1)
    y0 = torch.empty(0, dtype=torch.int32, device=dev)
    y1 = torch.empty(0, dtype=torch.int32, device=dev)
    ms = _timed(lambda: F.dpf_eval(y0, masked, key, s0, 0, N_BITS, N_BITS, 1), dev, max(3, min(args.steps, 10)))
    F.dpf_eval(y1, masked, key, s1, 1, N_BITS, N_BITS, 1)
    ok = bool(torch.equal((y0 + y1).view(-1), torch.where(x == 0, beta, torch.zeros_like(beta))))
    key_bytes = key.numel()
    del alpha, beta, s0, s1, x, masked, key, y0, y1
    torch.cuda.empty_cache()
    ach = DPF_LOOKUPS_PER_ELEM * N / (ms / 1e3) / 1e9
    full = dpf_all_section(dev, args, peak_glookups)
    return {"workload": "plain DPF eval, 2^24 elements, n=32, Z_2^32 (uint32), groupSize 1, one party per step",
            "elements": N, "kernel_ms": ms, "value": N / (ms / 1e3) / 1e9, "unit": "Gelem/s",
            "aes_blocks_per_s": (N_BITS + 1) * N / (ms / 1e3), "key_bytes_per_element": key_bytes / N,
            "hbm_gbs": (key_bytes + N * (16 + 4 + 4)) / (ms / 1e3) / 1e9,
            "roofline": {"bound": "smem", "achieved": ach, "peak": peak_glookups, "unit": "Glookup/s",
                         "frac": ach / peak_glookups, "algorithmic_lookups_per_element": DPF_LOOKUPS_PER_ELEM},
            "shares_reconstruct": ok, "eval_all": full}


# Full-domain DPF per key at n = 16, groupSize 1, 32-bit output: 2^n - 1 node expansions of
# both children under one key schedule (40 + 18 shared first-round + 2 x 144 rounds 2-9 and
# last = 346 lookups) and 2^n leaf converts (40 + 148, as above).
DPF_ALL_N = 16
DPF_ALL_LOOKUPS_PER_KEY = ((1 << DPF_ALL_N) - 1) * 346 + (1 << DPF_ALL_N) * (40 + 148)


def dpf_all_section(dev, args, peak_glookups) -> dict:
    """Full-domain DPF evaluation (FastFss_cuda_dpfEvalAll): 2^12 keys (--dpf-all-keys) at
    n = 16 over Z_2^32 (uint32), groupSize 1, every key expanded to its 2^16 outputs (1 GiB of
    shares per party at 2^12 keys)."""
    import torch

    import fastfunctionsecretsharing_b200 as F

    n, N = DPF_ALL_N, args.dpf_all_keys
    gen = torch.Generator(device=dev).manual_seed(8765)
    alpha = torch.randint(0, 1 << n, (N,), dtype=torch.int32, device=dev, generator=gen)
    beta = torch.randint(-2**31, 2**31, (N,), dtype=torch.int32, device=dev, generator=gen)
    s0 = torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device=dev, generator=gen)
    s1 = torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device=dev, generator=gen)
    x = torch.randint(0, 1 << n, (N,), dtype=torch.int32, device=dev, generator=gen)
    masked = (x + alpha) & ((1 << n) - 1)
    key = torch.empty(0, dtype=torch.uint8, device=dev)
    F.dpf_key_gen(key, alpha, beta, s0, s1, n, 32, 1)
    y0 = torch.empty(0, dtype=torch.int32, device=dev)
    y1 = torch.empty(0, dtype=torch.int32, device=dev)
    ms = _timed(lambda: F.dpf_eval_all(y0, masked, key, s0, 0, n, 32, 1), dev, max(3, min(args.steps, 10)))
    F.dpf_eval_all(y1, masked, key, s1, 1, n, 32, 1)
    # out[i][(maskedX - j) mod 2^n] = share of beta [j == alpha]: the reconstruction holds beta at x
    want = torch.zeros(N, 1 << n, dtype=torch.int32, device=dev)
    want[torch.arange(N, device=dev), x.long()] = beta
    ok = bool(torch.equal((y0 + y1).view(N, 1 << n), want))
    out_bytes = y0.numel() * 4
    del alpha, beta, s0, s1, x, masked, key, y0, y1, want
    torch.cuda.empty_cache()
    ach = DPF_ALL_LOOKUPS_PER_KEY * N / (ms / 1e3) / 1e9
    return {"workload": f"full-domain DPF eval, {N} keys, n=16, Z_2^32 (uint32), groupSize 1, one party per step",
            "keys": N, "kernel_ms": ms, "Gout_per_s": N * (1 << n) / (ms / 1e3) / 1e9,
            "out_gbs": out_bytes / (ms / 1e3) / 1e9,
            "roofline": {"bound": "smem", "achieved": ach, "peak": peak_glookups, "unit": "Glookup/s",
                         "frac": ach / peak_glookups, "algorithmic_lookups_per_key": DPF_ALL_LOOKUPS_PER_KEY},
            "shares_reconstruct": ok}


def grotto_section(dev, args, peak_glookups) -> dict:
    """Grotto full domain over Z_2: 2^16 keys at n = 16 expanded to 2^16 leaf bits each (equality
    rows and prefix-parity comparison rows, bit-packed), then a 64-segment lookup table (sorted
    random boundaries, 16-bit values) evaluated from the comparison rows with warp ballots and
    population counts; the same table through per-interval tree walks for comparison."""
    import numpy as np
    import torch

    import fastfunctionsecretsharing_b200 as F
    from fastfunctionsecretsharing_b200 import workloads as W

    n, es, N, m = 16, 2, 1 << 16, 64
    gen = torch.Generator(device=dev).manual_seed(99)
    rng = np.random.default_rng(99)
    alpha = torch.randint(-2**15, 2**15, (N,), dtype=torch.int16, device=dev, generator=gen)
    s0 = torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device=dev, generator=gen)
    s1 = torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device=dev, generator=gen)
    x = torch.randint(-2**15, 2**15, (N,), dtype=torch.int16, device=dev, generator=gen)
    masked = x + alpha
    key = torch.empty(0, dtype=torch.uint8, device=dev)
    F.grotto_key_gen(key, alpha, s0, s1, n)
    L, R = W.partition(rng, m, n)
    Lt, Rt = W._ring_tensor(L, es, dev), W._ring_tensor(R, es, dev)
    lut = torch.randint(-2**15, 2**15, (m,), dtype=torch.int16, device=dev, generator=gen)
    rows = torch.empty(N * ((1 << n) // 8), dtype=torch.uint8, device=dev)
    rows1 = torch.empty_like(rows)
    steps = max(3, min(args.steps, 10))
    e = [torch.empty(0, dtype=torch.int16, device=dev) for _ in range(4)]
    t = [torch.empty(0, dtype=torch.int16, device=dev) for _ in range(4)]

    eq_ms = _timed(lambda: F.grotto_eq_eval_all(rows, key, s0, 0, n, es, N), dev, steps)
    le_ms = _timed(lambda: F.grotto_le_eval_all(rows, key, s0, 0, n, es, N), dev, steps)
    lut_rows_ms = _timed(lambda: F.grotto_interval_lut_eval_from_rows(e[0], t[0], masked, rows, 0, Lt, Rt, lut, n),
                         dev, steps)
    walk_ms = _timed(lambda: F.grotto_interval_lut_eval(e[1], t[1], masked, key, s0, 0, Lt, Rt, lut, n, n), dev,
                     steps)
    same_as_walks = bool(torch.equal(e[0], e[1]) and torch.equal(t[0], t[1]))
    # party 1, then reconstruction as the reference's tests do it: E = E0 + E1 is +-1 (one
    # segment holds x), T = T0 + T1, and E * T = lut[segment of x]
    F.grotto_le_eval_all(rows1, key, s1, 1, n, es, N)
    F.grotto_interval_lut_eval_from_rows(e[2], t[2], masked, rows1, 1, Lt, Rt, lut, n)
    xs = x.to(torch.int64) & 0xFFFF
    seg = torch.searchsorted(torch.tensor(R, dtype=torch.int64, device=dev), xs)
    E = (e[0] + e[2]).view(-1)
    ok = bool((E.abs() == 1).all() and torch.equal(E * (t[0] + t[2]).view(-1), lut[seg]))
    del rows, rows1, key
    torch.cuda.empty_cache()
    # every internal node of the depth-(n-6) tree expanded once: key schedule + both children
    # (40 + 320) less the 14 first-round lookups they share; the parents of leaves skip the 4
    # last-round lookups of word 1 in each child (no leaf reads it)
    D = n - 6
    lookups_per_key = ((1 << (D - 1)) - 1) * 346 + (1 << (D - 1)) * 338
    ach = lookups_per_key * N / (le_ms / 1e3) / 1e9
    total = le_ms + lut_rows_ms
    return {"workload": ("Grotto full domain over Z_2: 2^16 keys, n=16 (2^16 leaf bits per key, bit-packed), then "
                         "a 64-segment LUT (sorted random boundaries, 16-bit values) by prefix parity"),
            "keys": N, "eq_rows_ms": eq_ms, "le_rows_ms": le_ms, "lut_from_rows_ms": lut_rows_ms,
            "lut_total_ms": total, "lut_by_walks_ms": walk_ms,
            "keys_per_s": N / (total / 1e3), "leaf_bits_per_s": N * (1 << n) / (le_ms / 1e3),
            "rows_gbs": N * (1 << n) / 8 / (le_ms / 1e3) / 1e9,
            "roofline_rows": {"bound": "smem", "achieved": ach, "peak": peak_glookups, "unit": "Glookup/s",
                              "frac": ach / peak_glookups, "algorithmic_lookups_per_key": lookups_per_key},
            "lut_same_as_walks": same_as_walks, "shares_reconstruct": ok}


def batched_section(dev, args, peak_glookups) -> dict:
    """Mixed-bitwidth MIC + spline batch: plain per-call C-ABI loop vs one persistent launch
    (autotuned, CUDA-graph captured), same instances, same stream; elements/s of both."""
    import torch

    from fastfunctionsecretsharing_b200 import batch as B
    from fastfunctionsecretsharing_b200 import workloads as W

    mic_log2, spline_log2 = (8, 18), (8, 13)
    inst = W.mixed_mic_spline(device=dev, instances=args.batched_instances, seed=4, mic_log2=mic_log2,
                              spline_log2=spline_log2)
    elems = sum(i.N for i in inst)
    lookups = sum(i.lookups for i in inst)
    stream = torch.cuda.current_stream(dev)
    steps = max(3, min(args.steps, 10))

    def timed(fn):
        for _ in range(2):
            fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / steps

    plain_ms = timed(lambda: W.run_plain(inst))
    b = B.Batch([i.request for i in inst], dev)
    best, timings = B.autotune(b, reps=2)
    g = b.graph()
    batched_ms = timed(g.replay)
    same = all(torch.equal(i.request.tensors[0].view(-1), i.out_plain.view(-1)) for i in inst)
    res = {"workload": (f"{args.batched_instances} instances: half DCF-MIC (16 sorted intervals, n in "
                        "{8,12,16,24,32,64}, N log-uniform 2^8..2^18), half spline (32 intervals, degree 2, "
                        "n=bo=64, N log-uniform 2^8..2^13); one party; keys device-resident"),
           "elements_per_step": elems, "plain_ms": plain_ms, "batched_ms": batched_ms,
           "plain_elem_per_s": elems / (plain_ms / 1e3), "batched_elem_per_s": elems / (batched_ms / 1e3),
           "speedup": plain_ms / batched_ms, "plain_launches_per_step": len(inst),
           "batched_launches_per_step": 1, "tuning": list(best.as_tuple()),
           "autotune_ms": {str(k): v for k, v in timings.items()}, "outputs_match_plain": bool(same),
           "algorithmic_lookups_per_step": lookups,
           "roofline": {"bound": "smem", "peak": peak_glookups, "unit": "Glookup/s",
                        "plain_frac": lookups / (plain_ms / 1e3) / 1e9 / peak_glookups,
                        "batched_frac": lookups / (batched_ms / 1e3) / 1e9 / peak_glookups}}
    del inst, b, g
    torch.cuda.empty_cache()
    return res


def serving_section(dev, args) -> dict:
    """Continuous-batching server vs plain per-call serving on the same Poisson arrivals."""
    import torch

    from fastfunctionsecretsharing_b200 import serving as S

    P = S.make_pools(dev, dcf_log2=(10, 20), spline_log2=(10, 14))
    out = {"workload": ("12-layer MLP (width 4096, batch 64) trace: 2^18 ReLU DCFs (n=32) + 2^18 GeLU splines "
                        "(n=64, 32 intervals, degree 2) per layer, issued as requests of 2^k elements (DCF k in "
                        "10..20, spline k in 10..14); key store 64 GB charged per request; batches capped at about "
                        "4 ms of GPU work, a new batch queued while under two batches of estimated work are in flight on "
                        "one stream; plain = one per-call C-ABI "
                        "evaluation per request, FIFO on one stream"),
           "rates": []}
    S.Server(P).warmup()
    for rate in (100.0, 1000.0, 10000.0):
        row = {"rate_req_per_s": rate}
        for mode in ("batched", "plain"):
            reqs = S.make_requests(P, rate=rate, count=args.serving_requests, seed=int(rate))
            srv = S.Server(P, capacity_bytes=64 << 30)
            makespan = srv.run(reqs, mode=mode)
            st = S.summarize(reqs, makespan)
            st["launches"] = srv.launches
            st["key_store_peak_gb"] = srv.store.peak / 2**30
            row[mode] = st
        out["rates"].append(row)
    del P
    torch.cuda.empty_cache()
    return out


def seed1_regen(gen_seed: int, N: int, dev):
    """Regenerates party 1's seeds exactly as the set-up drew them (same generator order)."""
    import torch

    gen = torch.Generator(device=dev).manual_seed(gen_seed)
    torch.randint(-2**31, 2**31, (N,), dtype=torch.int32, device=dev, generator=gen)
    torch.randint(-2**31, 2**31, (N,), dtype=torch.int32, device=dev, generator=gen)
    torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device=dev, generator=gen)
    return torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device=dev, generator=gen)


def FastFssSm(lib) -> int:
    return int(lib.fn("FastFss_b200_smCount")())


if __name__ == "__main__":
    main()
