"""Seeded synthetic workloads shared by the benchmark, the serving simulator and the tests.

``mixed_mic_spline`` builds the mixed-bitwidth batch: half DCF-based MIC instances (16 sorted
intervals, input width drawn from {8, 12, 16, 24, 32, 64}), half degree-2 splines (32
intervals over Z_2^64, fixed-point coefficients round(U[-4, 4) * 2^16) mod 2^64), element
counts log-uniform. Keys are generated on the device with this library's key generation;
inputs are uniform. Each instance yields a batch request and the equivalent plain per-call
invocation of the C ABI (prebuilt ctypes arguments, so the loop measures the library, not
Python).
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib, batch
from . import dcf_mic_key_gen, spline_get_cache_data_size, spline_key_gen

WIDTHS = (8, 12, 16, 24, 32, 64)
TORCH_DT = {1: torch.int8, 2: torch.int16, 4: torch.int32, 8: torch.int64}


def elem_size(n: int) -> int:
    return 1 if n <= 8 else 2 if n <= 16 else 4 if n <= 32 else 8


def _rand_ring(gen, shape, es, dev):
    if es == 8:
        return torch.randint(-2**63, 2**63 - 1, shape, dtype=torch.int64, device=dev, generator=gen)
    lo = -(1 << (8 * es - 1))
    return torch.randint(lo, -lo, shape, dtype=torch.int64, device=dev, generator=gen).to(TORCH_DT[es])


def _mask_bits(t: torch.Tensor, n: int) -> torch.Tensor:
    if n >= 8 * t.element_size():
        return t
    return t & ((1 << n) - 1)


def sorted_intervals(rng: np.random.Generator, m: int, n: int):
    """m intervals with sorted endpoints: boundaries b_0 < ... < b_m drawn uniformly, interval
    q = [b_q, b_{q+1} - 1] (touching intervals, as the reference's MIC tests draw them)."""
    dom = 1 << n
    pts: set[int] = set()
    while len(pts) < min(m + 1, dom):
        v = (int(rng.integers(0, 2**62)) * 4 + int(rng.integers(0, 4))) % dom
        pts.add(v)
    b = sorted(pts)
    L = b[:-1]
    R = [v - 1 for v in b[1:]]
    return L, R


def partition(rng: np.random.Generator, m: int, n: int):
    """m intervals covering [0, 2^n) with sorted random cut points, L_0 = 0."""
    dom = 1 << n
    cuts: set[int] = set()
    while len(cuts) < m - 1:
        v = (int(rng.integers(0, 2**62)) * 4 + int(rng.integers(0, 4))) % dom
        if v:
            cuts.add(v)
    L = [0] + sorted(cuts)
    R = [v - 1 for v in L[1:]] + [dom - 1]
    return L, R


def _ring_tensor(vals, es, dev):
    arr = np.array([v % (1 << (8 * es)) for v in vals], dtype=np.uint64).astype({1: np.uint8, 2: np.uint16,
                                                                              4: np.uint32, 8: np.uint64}[es])
    return torch.from_numpy(arr.view({1: np.int8, 2: np.int16, 4: np.int32, 8: np.int64}[es]).copy()).to(dev)


def dcf_level_lookups(bo: int) -> int:
    """AES table lookups of one groupSize-1 DCF level: key schedule (40), the seed child (160) and
    the value child less the 14 first-round lookups it shares with the seed child and the
    last-round columns a ceil(bo/8)-byte read does not need (4 per unused column)."""
    cols = 1 if (bo + 7) // 8 <= 4 else 2
    return 40 + 160 + 160 - 14 - 4 * (4 - cols)


def spline_window_blocks(m: int, cn: int, c0: int, cnt: int, ges: int) -> int:
    """Convert-stream blocks read per level for coefficients c0 .. c0 + cnt - 1 of an interval
    (the maximum over the intervals' byte offsets, as the kernels use it)."""
    nb = 1
    for q in range(min(m, 16)):
        off = ((q * cn + c0) * ges) & 15
        nb = max(nb, (off + cnt * ges + 15) >> 4)
    return nb


def algorithmic_lookups(kind: str, N: int, n: int, bo: int, m: int = 0, d: int = 0, tiling: bool = False) -> int:
    """AES table lookups one party's evaluation needs.

    mic: 2 m groupSize-1 DCF walks of n levels per element; with `tiling` (here: touching
    intervals, R_q + 1 = L_{q+1}) each of the m + 1 endpoint points is walked once.
    spline: per element and interval, two DCF walks of n levels; a level is the node expansion
    (key schedule + seed child + full value child, 346) and the convert of interval q's d + 1
    values out of the value child's AES-CTR stream (key schedule + the blocks holding them);
    the leaf adds one more convert per walk. Values are read 4 at a time. With `tiling`
    (intervals that tile the ring, R_{q-1} + 1 = L_q) the left endpoint of interval q is the
    right endpoint of interval q - 1: one walk per interval, whose converts read two slot
    windows (slots q and q - 1) under one key schedule."""
    if kind == "mic":
        walks = (m + 1) if tiling else 2 * m
        return N * walks * n * dcf_level_lookups(bo)
    if kind == "spline":
        cn, ges = d + 1, (bo + 7) // 8
        g = m * cn
        windows = 2 if tiling else 1
        conv = 0
        for c0 in range(0, cn, 4):
            cnt = min(4, cn - c0)
            conv += (40 + 160 * windows * spline_window_blocks(m, cn, c0, cnt, ges)) if ges * g > 16 else 0
        steps = 1 + (cn - 1) // 4  # the walks are repeated per pass of 4 coefficients
        walks = 1 if tiling else 2
        return N * m * walks * (steps * n * 346 + (n + 1) * conv)
    raise ValueError(kind)


@dataclass
class Instance:
    kind: str
    n: int
    es: int
    N: int
    request: batch.Request
    plain: tuple  # (ctypes function, argument tuple) of the per-call C ABI evaluation
    out_plain: torch.Tensor
    key_bytes: int
    lookups: int = 0  # algorithmic AES table lookups of one evaluation


def _stream_arg(dev):
    h = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    return h


def mixed_mic_spline(device="cuda", instances=256, seed=4, mic_log2=(8, 18), spline_log2=(8, 13),
                     mic_intervals=16, spline_intervals=32, degree=2, party=0) -> list[Instance]:
    dev = torch.device(device)
    rng = np.random.default_rng(seed)
    gen = torch.Generator(device=dev).manual_seed(seed)
    stream_h = _stream_arg(dev)
    out: list[Instance] = []
    for k in range(instances):
        spline = k % 2 == 1
        if spline:
            n = bo = 64
            lo, hi = spline_log2
        else:
            n = bo = int(rng.choice(WIDTHS))
            lo, hi = mic_log2
        es = elem_size(n)
        N = int(round(2 ** rng.uniform(lo, hi)))
        alpha = _mask_bits(_rand_ring(gen, (N,), es, dev), n)
        s0 = torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device=dev, generator=gen)
        s1 = torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device=dev, generator=gen)
        x = _mask_bits(_rand_ring(gen, (N,), es, dev), n)
        masked = _mask_bits(x + alpha, n)
        seed_p = s0 if party == 0 else s1
        if not spline:
            L, R = sorted_intervals(rng, mic_intervals, n)
            Lt, Rt = _ring_tensor(L, es, dev), _ring_tensor(R, es, dev)
            key = torch.empty(0, dtype=torch.uint8, device=dev)
            z = torch.empty(0, dtype=TORCH_DT[es], device=dev)
            dcf_mic_key_gen(key, z, alpha, s0, s1, Lt, Rt, n, bo)
            zs = _rand_ring(gen, z.shape, es, dev)  # party-0 share of z (party 1 holds z - zs)
            if party == 1:
                zs = z - zs
            o_b = torch.empty(0, dtype=TORCH_DT[es], device=dev)
            req = batch.mic_request(o_b, masked, key, zs, seed_p, party, Lt, Rt, n, bo)
            o_p = torch.empty((N, mic_intervals), dtype=TORCH_DT[es], device=dev)
            fn = _lib.fn("FastFss_cuda_dcfMICEval")
            args = (o_p.data_ptr(), o_p.numel() * es, masked.data_ptr(), N * es, key.data_ptr(), key.numel(),
                    zs.data_ptr(), zs.numel() * es, seed_p.data_ptr(), N * 16, party, Lt.data_ptr(), Lt.numel() * es,
                    Rt.data_ptr(), Rt.numel() * es, n, bo, es, N, None, 0, ctypes.byref(stream_h))
            req.tensors += [o_p]
            out.append(Instance("mic", n, es, N, req, (fn, args), o_p, key.numel(),
                                algorithmic_lookups("mic", N, n, bo, mic_intervals, tiling=True)))
        else:
            m, d = spline_intervals, degree
            L, R = partition(rng, m, n)
            Lt, Rt = _ring_tensor(L, es, dev), _ring_tensor(R, es, dev)
            coeffs = [int(round(rng.uniform(-4, 4) * 65536)) for _ in range(m * (d + 1))]
            ct = _ring_tensor(coeffs, es, dev)
            key = torch.empty(0, dtype=torch.uint8, device=dev)
            e = torch.empty(0, dtype=TORCH_DT[es], device=dev)
            beta = torch.empty(0, dtype=TORCH_DT[es], device=dev)
            spline_key_gen(key, e, beta, alpha, s0, s1, ct, d, Lt, Rt, m, n, bo)
            es0 = _rand_ring(gen, e.shape, es, dev)
            b0 = _rand_ring(gen, beta.shape, es, dev)
            if party == 1:
                es0, b0 = e - es0, beta - b0
            o_b = torch.empty(0, dtype=TORCH_DT[es], device=dev)
            req = batch.spline_request(o_b, masked, key, es0, b0, seed_p, party, Lt, Rt, m, d, n, bo)
            o_p = torch.empty((N,), dtype=TORCH_DT[es], device=dev)
            csize = spline_get_cache_data_size(d, m, n, bo, es, N)
            cache = torch.empty(csize, dtype=torch.uint8, device=dev)
            fn = _lib.fn("FastFss_cuda_dcfSplineEval")
            args = (o_p.data_ptr(), N * es, masked.data_ptr(), N * es, key.data_ptr(), key.numel(), es0.data_ptr(),
                    es0.numel() * es, b0.data_ptr(), b0.numel() * es, seed_p.data_ptr(), N * 16, party, Lt.data_ptr(),
                    m * es, Rt.data_ptr(), m * es, m, d, n, bo, es, N, cache.data_ptr(), csize,
                    ctypes.byref(stream_h))
            req.tensors += [o_p, cache]
            out.append(Instance("spline", n, es, N, req, (fn, args), o_p, key.numel(),
                                algorithmic_lookups("spline", N, n, bo, m, d, tiling=True)))
        del s0, s1
    torch.cuda.synchronize(dev)
    return out


def run_plain(instances: list[Instance]) -> None:
    for inst in instances:
        fn, args = inst.plain
        rc = fn(*args)
        if rc != 0:
            raise RuntimeError(f"plain call failed : {rc}")


def log_uniform_sizes(rng, count, lo, hi):
    return [int(round(2 ** rng.uniform(lo, hi))) for _ in range(count)]


def mean_log_uniform(lo, hi):
    return (2 ** hi - 2 ** lo) / ((hi - lo) * math.log(2))
