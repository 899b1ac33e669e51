"""Continuous-batching FSS evaluation server, driven by a simulated two-party inference engine.

The engine runs a 12-layer MLP (width 4096, batch 64); every layer needs 2^18 ReLU
comparisons (DCF, n = 32 over Z_2^32) and 2^18 GeLU splines (32 intervals, degree 2,
n = 64 over Z_2^64). It issues that work as requests of 2^k elements (k uniform), arriving
as a Poisson process. The server

* keeps key material device-resident in a key store whose capacity is counted in bytes; a
  request is admitted only when its keys fit in the remaining capacity (charged on
  admission, released on completion);
* batches continuously: admitted requests are taken from the head of the FIFO queue into one
  persistent batched launch until the batch's estimated GPU time (algorithmic AES lookups at
  the lookup rate of the kernels) reaches `batch_cap_ms`, so early arrivals are not held back
  behind everything queued after them; a new batch is queued (on the stream slots in turn; one
  slot by default, as every batch spans all SMs) while the launches still queued or running
  hold less than `max_inflight` batches' worth of estimated GPU time (a launch counts in full
  until it completes, so the next round is queued behind a long launch instead of after it),
  so the device never idles between batches (a count of launches would let a queue that ends
  in a few tiny launches drain) and a request waits behind a bounded amount of work. Within a batch, requests that fill every SM
  on their own (DCF requests of >= 148 x 512 elements, spline requests of >= 148 x 16) go out
  as their own per-call launches in queue order, and only the runs of smaller requests share a
  persistent batched launch (that is where one launch gains: small requests cannot fill the
  GPU, while a large one is served best by its dedicated kernel). A request's
  masked input is copied in from pinned host memory and its shares copied back on the same
  stream;
* records per-request latency (completion - arrival, wall clock; completion is observed by
  polling the launch's CUDA event).

The `plain` mode serves the same arrivals without batching: every admitted request is its own
per-call C-ABI evaluation, queued FIFO on one stream (the spline cache the per-call API
requires is allocated once per size class, not per call).

Key material: the store charges every request its key bytes; the kernels read valid keys from
one pool per kind and size class, so every evaluation is real and checkable while the 64 GB
model stays within one GPU.
"""

from __future__ import annotations

import ctypes
import gc
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib, batch
from . import dcf_key_gen, spline_get_cache_data_size, spline_key_gen
from .workloads import _rand_ring, _ring_tensor, algorithmic_lookups, dcf_level_lookups, partition

DCF_N = 32
SPLINE_N, SPLINE_M, SPLINE_D = 64, 32, 2
SPLINE_G = SPLINE_M * (SPLINE_D + 1)
DCF_KEY_BYTES = 16 * DCF_N + 4 * DCF_N + 3 * 4  # per element (652)
SPLINE_KEY_BYTES = 16 * SPLINE_N + 8 * SPLINE_N * SPLINE_G + 2 * 8 + 8 * SPLINE_G  # per element (50,960)


@dataclass
class Request:
    rid: int
    kind: str  # "dcf" or "spline"
    layer: int
    size: int
    arrival: float
    key_bytes: int
    start: float = 0.0
    done: float = 0.0
    x_host: torch.Tensor | None = None
    out_host: torch.Tensor | None = None
    x_dev: torch.Tensor | None = None    # the request's device buffers, allocated before serving
    out_dev: torch.Tensor | None = None  # starts (nothing is allocated while requests are served)


@dataclass
class SizeClass:
    """Valid keys (and the other per-element key material) for requests of N elements."""

    N: int
    key: torch.Tensor
    seed: torch.Tensor
    e: torch.Tensor | None = None
    beta: torch.Tensor | None = None
    cache: torch.Tensor | None = None  # the spline eval cache the per-call API requires (reused)


@dataclass
class Pools:
    dev: torch.device
    party: int
    dcf: dict = field(default_factory=dict)
    spline: dict = field(default_factory=dict)
    spline_L: torch.Tensor | None = None
    spline_R: torch.Tensor | None = None


def make_pools(device, dcf_log2=(10, 20), spline_log2=(10, 14), seed=9, party=0) -> Pools:
    """Generates (on the device) keys for every power-of-two request size."""
    dev = torch.device(device)
    gen = torch.Generator(device=dev).manual_seed(seed)
    rng = np.random.default_rng(seed)
    P = Pools(dev, party)
    for k in range(dcf_log2[0], dcf_log2[1] + 1):
        N = 1 << k
        a, b = _rand_ring(gen, (N,), 4, dev), _rand_ring(gen, (N,), 4, dev)
        s0 = torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device=dev, generator=gen)
        s1 = torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device=dev, generator=gen)
        key = torch.empty(0, dtype=torch.uint8, device=dev)
        dcf_key_gen(key, a, b, s0, s1, DCF_N, DCF_N, 1)
        P.dcf[N] = SizeClass(N, key, s0 if party == 0 else s1)
    L, R = partition(rng, SPLINE_M, SPLINE_N)
    P.spline_L, P.spline_R = _ring_tensor(L, 8, dev), _ring_tensor(R, 8, dev)
    coeffs = [int(round(rng.uniform(-4, 4) * 65536)) for _ in range(SPLINE_G)]
    ct = _ring_tensor(coeffs, 8, dev)
    for k in range(spline_log2[0], spline_log2[1] + 1):
        N = 1 << k
        a = _rand_ring(gen, (N,), 8, dev)
        s0 = torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device=dev, generator=gen)
        s1 = torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device=dev, generator=gen)
        key = torch.empty(0, dtype=torch.uint8, device=dev)
        e = torch.empty(0, dtype=torch.int64, device=dev)
        beta = torch.empty(0, dtype=torch.int64, device=dev)
        spline_key_gen(key, e, beta, a, s0, s1, ct, SPLINE_D, P.spline_L, P.spline_R, SPLINE_M, SPLINE_N, SPLINE_N)
        e0, b0 = _rand_ring(gen, e.shape, 8, dev), _rand_ring(gen, beta.shape, 8, dev)
        if party == 1:
            e0, b0 = e - e0, beta - b0
        cache = torch.empty(spline_get_cache_data_size(SPLINE_D, SPLINE_M, SPLINE_N, SPLINE_N, 8, N),
                            dtype=torch.uint8, device=dev)
        P.spline[N] = SizeClass(N, key, s0 if party == 0 else s1, e0, b0, cache)
    torch.cuda.synchronize(dev)
    return P


class KeyStore:
    """Device-resident key budget; a request's keys are charged on admission."""

    def __init__(self, capacity_bytes: int):
        self.capacity = capacity_bytes
        self.used = 0
        self.peak = 0

    def try_admit(self, nbytes: int) -> bool:
        if self.used + nbytes > self.capacity:
            return False
        self.used += nbytes
        self.peak = max(self.peak, self.used)
        return True

    def release(self, nbytes: int) -> None:
        self.used -= nbytes


def mlp_trace(rng: np.random.Generator, layers=12, width=4096, batch_rows=64, lo=10, hi=20, spline_hi=14,
              limit: int | None = None):
    """Splits every layer's width * batch_rows DCF and spline evaluations into requests of 2^k
    elements, k uniform in [lo, hi] (spline: [lo, spline_hi]), alternating the two kinds."""
    per_layer = width * batch_rows
    reqs = []
    for layer in range(layers):
        left = {"dcf": per_layer, "spline": per_layer}
        while left["dcf"] > 0 or left["spline"] > 0:
            for kind, top in (("dcf", hi), ("spline", min(hi, spline_hi))):
                if left[kind] <= 0:
                    continue
                size = 1 << int(rng.integers(lo, top + 1))
                while size > left[kind]:
                    size >>= 1
                reqs.append((kind, layer, size))
                left[kind] -= size
                if limit and len(reqs) >= limit:
                    return reqs
    return reqs


def make_requests(P: Pools, rate: float, count: int, seed: int = 1, dcf_log2=(10, 20), spline_log2=(10, 14)):
    """`count` requests of the MLP trace with Poisson arrivals at `rate` per second (arrival
    times relative to the start). Host inputs and outputs are pinned; each request's device
    input and output buffers are allocated here too, so that serving itself allocates nothing
    (an allocation that has to free cached device memory synchronises the whole device)."""
    rng = np.random.default_rng(seed)
    trace = mlp_trace(rng, lo=dcf_log2[0], hi=dcf_log2[1], spline_hi=spline_log2[1], limit=count)
    t = 0.0
    out = []
    for rid, (kind, layer, size) in enumerate(trace[:count]):
        t += rng.exponential(1.0 / rate)
        if kind == "dcf":
            xb = torch.from_numpy(rng.integers(-2**31, 2**31, size=size, dtype=np.int64).astype(np.int32)).pin_memory()
            ob = torch.empty(size, dtype=torch.int32).pin_memory()
            kb = size * DCF_KEY_BYTES
        else:
            xb = torch.from_numpy(rng.integers(-2**63, 2**63 - 1, size=size, dtype=np.int64)).pin_memory()
            ob = torch.empty(size, dtype=torch.int64).pin_memory()
            kb = size * SPLINE_KEY_BYTES
        dt = torch.int32 if kind == "dcf" else torch.int64
        out.append(Request(rid, kind, layer, size, t, kb, x_host=xb, out_host=ob,
                           x_dev=torch.empty(size, dtype=dt, device=P.dev),
                           out_dev=torch.empty(size, dtype=dt, device=P.dev)))
    return out


# Estimated evaluation cost (AES table lookups) per element, used to cap a batch's GPU time.
DCF_LOOKUPS = DCF_N * dcf_level_lookups(DCF_N)
SPLINE_LOOKUPS = algorithmic_lookups("spline", 1, SPLINE_N, SPLINE_N, SPLINE_M, SPLINE_D, tiling=True)


def request_lookups(r: Request) -> int:
    return r.size * (DCF_LOOKUPS if r.kind == "dcf" else SPLINE_LOOKUPS)


class Server:
    MAX_BATCH_OPS = 4096  # requests per batch that fit the preallocated workspace
    def __init__(self, pools: Pools, capacity_bytes=64 << 30, slots=1, tuning: batch.Tuning | None = None,
                 max_inflight: int = 2, batch_cap_ms: float = 4.0, lookups_per_s: float = 8.0e12):
        self.P = pools
        self.dev = pools.dev
        self.store = KeyStore(capacity_bytes)
        self.slots = [torch.cuda.Stream(self.dev) for _ in range(slots)]
        # one batch workspace per stream slot (batches on a slot run in order), so serving
        # allocates nothing per batch
        self.workspaces = [torch.empty(batch.workspace_size(self.MAX_BATCH_OPS), dtype=torch.uint8, device=self.dev)
                           for _ in range(slots)]
        self.tuning = tuning  # None: per batch, see _tuning_for
        self.max_inflight = max(1, max_inflight)
        self.batch_cap = batch_cap_ms * 1e-3 * lookups_per_s
        self.launches = 0
        self.batch_log: list | None = None  # set to [] to record per-batch host time and kernel events
        self.sm_threads = torch.cuda.get_device_properties(self.dev).multi_processor_count * 512

    def warmup(self) -> None:
        """One request of every size class through both paths, synchronously: loads the kernels
        and fills the allocator's caches before anything is timed."""
        reqs = []
        for kind, pool in (("dcf", self.P.dcf), ("spline", self.P.spline)):
            for n in pool:
                dt = torch.int32 if kind == "dcf" else torch.int64
                reqs.append(Request(-1, kind, 0, n, 0.0, 0, x_host=torch.zeros(n, dtype=dt).pin_memory(),
                                    out_host=torch.empty(n, dtype=dt).pin_memory(),
                                    x_dev=torch.empty(n, dtype=dt, device=self.dev),
                                    out_dev=torch.empty(n, dtype=dt, device=self.dev)))
        s = self.slots[0]
        with torch.cuda.stream(s):
            for r in reqs:
                self._plain_call(r, s)
            built = [self._build(r) for r in reqs]
            batch.Batch(built, self.dev).prepare(self._tuning_for(reqs)).launch()
            batch.Batch(built[:1], self.dev).prepare(batch.Tuning(512, 1 << 26, 0, 0)).launch()
        torch.cuda.synchronize(self.dev)

    def _build(self, r: Request) -> batch.Request:
        """Device buffers and the batch request of r (input copied in on the current stream)."""
        P = self.P
        if r.kind == "dcf":
            c = P.dcf[r.size]
            x, out = r.x_dev, r.out_dev
            x.copy_(r.x_host, non_blocking=True)
            return batch.dcf_request(out, x, c.key, c.seed, P.party, DCF_N, DCF_N)
        c = P.spline[r.size]
        x, out = r.x_dev, r.out_dev
        x.copy_(r.x_host, non_blocking=True)
        return batch.spline_request(out, x, c.key, c.e, c.beta, c.seed, P.party, P.spline_L, P.spline_R, SPLINE_M,
                                    SPLINE_D, SPLINE_N, SPLINE_N)

    def _plain_call(self, r: Request, stream):
        """r alone through its per-call C-ABI entry point on `stream`."""
        P = self.P
        h = ctypes.c_void_p(stream.cuda_stream)
        if r.kind == "dcf":
            c = P.dcf[r.size]
            x, out = r.x_dev, r.out_dev
            x.copy_(r.x_host, non_blocking=True)
            rc = _lib.fn("FastFss_cuda_dcfEval")(out.data_ptr(), 4 * r.size, x.data_ptr(), 4 * r.size,
                                                c.key.data_ptr(), c.key.numel(), c.seed.data_ptr(), 16 * r.size,
                                                P.party, DCF_N, DCF_N, 1, 4, r.size, None, 0, ctypes.byref(h))
            keep = (x, out)
        else:
            c = P.spline[r.size]
            g = SPLINE_G
            x, out = r.x_dev, r.out_dev
            x.copy_(r.x_host, non_blocking=True)
            cache = c.cache
            csize = cache.numel()
            rc = _lib.fn("FastFss_cuda_dcfSplineEval")(
                out.data_ptr(), 8 * r.size, x.data_ptr(), 8 * r.size, c.key.data_ptr(), c.key.numel(),
                c.e.data_ptr(), 8 * g * r.size, c.beta.data_ptr(), 8 * g * r.size, c.seed.data_ptr(), 16 * r.size,
                P.party, P.spline_L.data_ptr(), 8 * SPLINE_M, P.spline_R.data_ptr(), 8 * SPLINE_M, SPLINE_M, SPLINE_D,
                SPLINE_N, SPLINE_N, 8, r.size, cache.data_ptr(), csize, ctypes.byref(h))
            keep = (x, out, cache)
        if rc != 0:
            raise RuntimeError(f"plain evaluation failed : {rc}")
        r.out_host.copy_(out.view(-1), non_blocking=True)
        return keep

    def run(self, requests: list[Request], mode: str = "batched", poll_s: float = 2e-5) -> float:
        """Serves `requests` in real time; returns the makespan in seconds. Python's cyclic
        garbage collector is paused meanwhile (a full collection over the pools' and requests'
        objects would stall the loop for tens of milliseconds)."""
        was = gc.isenabled()
        gc.disable()
        try:
            return self._run(requests, mode, poll_s)
        finally:
            if was:
                gc.enable()

    def _tuning_for(self, rs: list[Request]) -> batch.Tuning:
        """The server's tuning if it was given one; otherwise 256-thread CTAs for a batch with
        spline requests (the 512-thread persistent kernel must fit the spline path in 128
        registers and spills) and 512-thread CTAs for DCF-only batches."""
        if self.tuning is not None:
            return self.tuning
        threads = 256 if any(r.kind == "spline" for r in rs) else 512
        return batch.Tuning(threads, 1 << 26, 0, 0)

    def _fills_gpu(self, r: Request) -> bool:
        """True if r's own launch already puts a full CTA on every SM (a DCF element is one
        thread, a spline element one warp)."""
        return r.size * (1 if r.kind == "dcf" else 32) >= self.sm_threads

    def _launch_plain(self, r: Request, s, t0: float):
        with torch.cuda.stream(s):
            keep = self._plain_call(r, s)
            ev = torch.cuda.Event()
            ev.record(s)
        self.launches += 1
        r.start = time.perf_counter() - t0
        return ev, None, [r], keep

    def _launch_batch(self, rs: list[Request], si: int, t0: float):
        s = self.slots[si]
        h0 = time.perf_counter()
        with torch.cuda.stream(s):
            reqs = [self._build(r) for r in rs]
            b = batch.Batch(reqs, self.dev, workspace=self.workspaces[si]).prepare(self._tuning_for(rs))
            if self.batch_log is not None:
                e0 = torch.cuda.Event(enable_timing=True)
                e0.record(s)
            b.launch()
            if self.batch_log is not None:
                e1 = torch.cuda.Event(enable_timing=True)
                e1.record(s)
                self.batch_log.append({"requests": len(rs), "lookups": sum(request_lookups(r) for r in rs),
                                       "host_ms": (time.perf_counter() - h0) * 1e3, "events": (e0, e1)})
            for r, q in zip(rs, reqs):
                r.out_host.copy_(q.tensors[0].view(-1), non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(s)
        self.launches += 1
        tstart = time.perf_counter() - t0
        for r in rs:
            r.start = tstart
        return ev, si, rs, (b, reqs)

    def _run(self, requests: list[Request], mode: str, poll_s: float) -> float:
        pending: deque[Request] = deque()
        arrivals = deque(sorted(requests, key=lambda r: r.arrival))
        inflight = []  # (event, slot index or None, [requests], keep-alive, estimated lookups)
        outstanding = 0  # estimated lookups of the launches in flight
        done, total = 0, len(requests)
        t0 = time.perf_counter()
        while done < total:
            now = time.perf_counter() - t0
            while arrivals and arrivals[0].arrival <= now:
                pending.append(arrivals.popleft())
            still = []
            for entry in inflight:
                if entry[0].query():
                    tdone = time.perf_counter() - t0
                    for r in entry[2]:
                        r.done = tdone
                        self.store.release(r.key_bytes)
                    done += len(entry[2])
                    outstanding -= entry[4]
                else:
                    still.append(entry)
            inflight = still
            if mode == "batched":
                if pending and (not inflight or outstanding < self.max_inflight * self.batch_cap):
                    admitted, cost = [], 0
                    while pending and (not admitted or cost + request_lookups(pending[0]) <= self.batch_cap) \
                            and self.store.try_admit(pending[0].key_bytes):
                        cost += request_lookups(pending[0])
                        admitted.append(pending.popleft())
                    if admitted:
                        # FIFO order on one stream: runs of requests too small to fill the GPU
                        # share a persistent launch; a request that fills it alone takes its
                        # per-call kernel (the batched launch would add nothing but a slower
                        # generic kernel for it).
                        si = self.launches % len(self.slots)
                        run: list[Request] = []
                        for r in admitted + [None]:
                            if r is not None and not self._fills_gpu(r):
                                run.append(r)
                                continue
                            if run:
                                cost = sum(request_lookups(q) for q in run)
                                inflight.append((*self._launch_batch(run, si, t0), cost))
                                outstanding += cost
                                run = []
                            if r is not None:
                                inflight.append((*self._launch_plain(r, self.slots[si], t0), request_lookups(r)))
                                outstanding += request_lookups(r)
            else:
                while pending and self.store.try_admit(pending[0].key_bytes):
                    r = pending.popleft()
                    inflight.append((*self._launch_plain(r, self.slots[0], t0), request_lookups(r)))
                    outstanding += request_lookups(r)
            if not (arrivals and arrivals[0].arrival <= time.perf_counter() - t0):
                time.sleep(poll_s)
        return time.perf_counter() - t0


def summarize(reqs: list[Request], makespan: float) -> dict:
    lat = np.array([(r.done - r.arrival) * 1e3 for r in reqs])
    elems = sum(r.size for r in reqs)
    return {"requests": len(reqs), "elements": elems, "elements_per_s": elems / makespan, "makespan_s": makespan,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean())}


def reference_outputs(server: Server, reqs: list[Request]) -> list[np.ndarray]:
    """Each request evaluated alone through the per-call C ABI (the alone-vs-mix check)."""
    outs = []
    s = torch.cuda.current_stream(server.dev)
    for r in reqs:
        saved = r.out_host
        r.out_host = torch.empty_like(saved)
        server._plain_call(r, s)
        torch.cuda.synchronize(server.dev)
        outs.append(r.out_host.numpy().copy())
        r.out_host = saved
    return outs
