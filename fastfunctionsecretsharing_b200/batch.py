"""Batched evaluation: many FSS requests of mixed kinds and widths in one persistent launch.

Thin Python face of ``include/FastFss/b200/batch.h``: build ops from torch tensors, prepare a
plan (validation, tiling, descriptor upload into a device workspace), then launch — directly,
or captured once in a CUDA graph and replayed. ``autotune`` picks the launch shape (threads
per CTA, tile size, tile order) for a batch by timing the candidates on the device.
"""

from __future__ import annotations

import ctypes
import itertools
from ctypes import c_double, c_int32, c_uint32, c_uint64, c_void_p
from dataclasses import dataclass, field

import torch

from . import _lib

DCF_EVAL, DPF_EVAL, DCF_MIC_EVAL, SPLINE_EVAL, GROTTO_EVAL = 1, 2, 3, 4, 5


class BatchOp(ctypes.Structure):
    _fields_ = [("kind", c_int32), ("partyId", c_int32), ("elementSize", c_uint32), ("bitWidthIn", c_uint32),
                ("bitWidthOut", c_uint32), ("intervalNum", c_uint32), ("degree", c_uint32),
                ("equalBound", c_uint32), ("elementNum", c_uint64), ("sharedOut", c_void_p), ("maskedX", c_void_p),
                ("key", c_void_p), ("seed", c_void_p), ("aux0", c_void_p), ("aux1", c_void_p),
                ("leftEndpoints", c_void_p), ("rightEndpoints", c_void_p)]


class Tuning(ctypes.Structure):
    _fields_ = [("ctaThreads", c_uint32), ("tileLookups", c_uint32), ("order", c_uint32), ("reserved", c_uint32)]

    def as_tuple(self):
        return (self.ctaThreads, self.tileLookups, self.order)


class Plan(ctypes.Structure):
    _fields_ = [("totalTiles", c_uint64), ("totalItems", c_uint64), ("lookups", c_double), ("opNum", c_uint32),
                ("ctaThreads", c_uint32)]


_SIGS = {
    "FastFss_cuda_batchWorkspaceSize": (ctypes.c_size_t, [ctypes.c_size_t]),
    "FastFss_cuda_batchPrepare": (ctypes.c_int, [c_void_p, ctypes.c_size_t, c_void_p, c_void_p, ctypes.c_size_t,
                                                 c_void_p, c_void_p]),
    "FastFss_cuda_batchLaunch": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_size_t, c_void_p]),
}


def _fn(name):
    f = _lib.fn(name)
    res, args = _SIGS[name]
    f.restype, f.argtypes = res, args
    return f


def _p(t: torch.Tensor | None):
    return None if t is None else t.data_ptr()


@dataclass
class Request:
    """One evaluation request: the op plus the tensors it points at (kept alive)."""

    op: BatchOp
    tensors: list = field(default_factory=list)
    elements: int = 0


def dcf_request(out, maskedX, key, seed, partyId, bitWidthIn, bitWidthOut) -> Request:
    out.resize_(maskedX.shape + (1,))
    op = BatchOp(kind=DCF_EVAL, partyId=partyId, elementSize=maskedX.element_size(), bitWidthIn=bitWidthIn,
                 bitWidthOut=bitWidthOut, elementNum=maskedX.numel(), sharedOut=_p(out), maskedX=_p(maskedX),
                 key=_p(key), seed=_p(seed))
    return Request(op, [out, maskedX, key, seed], maskedX.numel())


def dpf_request(out, maskedX, key, seed, partyId, bitWidthIn, bitWidthOut) -> Request:
    out.resize_(maskedX.shape + (1,))
    op = BatchOp(kind=DPF_EVAL, partyId=partyId, elementSize=maskedX.element_size(), bitWidthIn=bitWidthIn,
                 bitWidthOut=bitWidthOut, elementNum=maskedX.numel(), sharedOut=_p(out), maskedX=_p(maskedX),
                 key=_p(key), seed=_p(seed))
    return Request(op, [out, maskedX, key, seed], maskedX.numel())


def mic_request(out, maskedX, key, sharedZ, seed, partyId, left, right, bitWidthIn, bitWidthOut) -> Request:
    out.resize_(maskedX.shape + (left.numel(),))
    op = BatchOp(kind=DCF_MIC_EVAL, partyId=partyId, elementSize=maskedX.element_size(), bitWidthIn=bitWidthIn,
                 bitWidthOut=bitWidthOut, intervalNum=left.numel(), elementNum=maskedX.numel(), sharedOut=_p(out),
                 maskedX=_p(maskedX), key=_p(key), seed=_p(seed), aux0=_p(sharedZ), leftEndpoints=_p(left),
                 rightEndpoints=_p(right))
    return Request(op, [out, maskedX, key, sharedZ, seed, left, right], maskedX.numel())


def spline_request(out, maskedX, key, sharedE, sharedBeta, seed, partyId, left, right, intervalNum, degree,
                   bitWidthIn, bitWidthOut) -> Request:
    out.resize_(maskedX.shape)
    op = BatchOp(kind=SPLINE_EVAL, partyId=partyId, elementSize=maskedX.element_size(), bitWidthIn=bitWidthIn,
                 bitWidthOut=bitWidthOut, intervalNum=intervalNum, degree=degree, elementNum=maskedX.numel(),
                 sharedOut=_p(out), maskedX=_p(maskedX), key=_p(key), seed=_p(seed), aux0=_p(sharedE),
                 aux1=_p(sharedBeta), leftEndpoints=_p(left), rightEndpoints=_p(right))
    return Request(op, [out, maskedX, key, sharedE, sharedBeta, seed, left, right], maskedX.numel())


def grotto_request(out, maskedX, key, seed, equalBound, partyId, bitWidthIn) -> Request:
    out.resize_(maskedX.shape)
    op = BatchOp(kind=GROTTO_EVAL, partyId=partyId, elementSize=maskedX.element_size(), bitWidthIn=bitWidthIn,
                 bitWidthOut=bitWidthIn, equalBound=int(bool(equalBound)), elementNum=maskedX.numel(),
                 sharedOut=_p(out), maskedX=_p(maskedX), key=_p(key), seed=_p(seed))
    return Request(op, [out, maskedX, key, seed], maskedX.numel())


def workspace_size(opNum: int) -> int:
    """Device bytes a batch of opNum ops needs (FastFss_cuda_batchWorkspaceSize)."""
    return int(_fn("FastFss_cuda_batchWorkspaceSize")(opNum))


class Batch:
    """A fixed set of requests, prepared once and launched any number of times."""

    def __init__(self, requests: list[Request], device: torch.device | str = "cuda",
                 workspace: torch.Tensor | None = None):
        """`workspace`: a device byte buffer to hold the queue counter and op table instead of a
        fresh allocation (at least workspace_size(len(requests)) bytes). Batches that share one
        must run on one stream, where each launch finishes before the next prepare's copy."""
        self.requests = list(requests)
        self.device = torch.device(device)
        self.ops = (BatchOp * max(1, len(self.requests)))(*[r.op for r in self.requests])
        n = len(self.requests)
        ws = workspace_size(n)
        if workspace is not None and workspace.numel() >= ws:
            self.workspace = workspace
        else:
            self.workspace = torch.empty(ws, dtype=torch.uint8, device=self.device)
        self.plan = Plan()
        self.tuning = Tuning(256, 1 << 26, 0, 0)
        self.elements = sum(r.elements for r in self.requests)

    def _stream_ref(self):
        h = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        return h, ctypes.byref(h)

    def prepare(self, tuning: Tuning | None = None) -> "Batch":
        if tuning is not None:
            self.tuning = tuning
        _, sref = self._stream_ref()
        rc = _fn("FastFss_cuda_batchPrepare")(ctypes.addressof(self.ops), len(self.requests),
                                               ctypes.byref(self.tuning), self.workspace.data_ptr(),
                                               self.workspace.numel(), ctypes.byref(self.plan), sref)
        if rc != 0:
            raise RuntimeError(f"FastFss_cuda_batchPrepare failed : {rc}")
        return self

    def launch(self) -> None:
        _, sref = self._stream_ref()
        rc = _fn("FastFss_cuda_batchLaunch")(ctypes.byref(self.plan), self.workspace.data_ptr(),
                                              self.workspace.numel(), sref)
        if rc != 0:
            raise RuntimeError(f"FastFss_cuda_batchLaunch failed : {rc}")

    def graph(self) -> torch.cuda.CUDAGraph:
        """Captures one launch (queue reset + persistent kernel) in a CUDA graph."""
        self.launch()  # sets the kernel's shared-memory attribute outside the capture
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.launch()
        return g


DEFAULT_CANDIDATES = [Tuning(t, tl, o, 0) for t, tl, o in itertools.product((256, 512), (1 << 24, 1 << 26, 1 << 28),
                                                                           (0, 1))]

_cache: dict[tuple, Tuning] = {}


def signature(batch: Batch) -> tuple:
    """Workload signature for the autotuner cache: kinds, widths and log2-sizes of the ops."""
    sig = []
    for r in batch.requests:
        o = r.op
        sig.append((o.kind, o.elementSize, o.bitWidthIn, o.intervalNum, o.degree, max(1, int(o.elementNum)).bit_length()))
    return tuple(sorted(sig))


def autotune(batch: Batch, candidates: list[Tuning] | None = None, reps: int = 3) -> tuple[Tuning, dict]:
    """Times every candidate launch shape on the device (CUDA events, after one warm-up) and
    prepares the batch with the fastest. Results are cached per workload signature."""
    sig = signature(batch)
    if sig in _cache:
        batch.prepare(_cache[sig])
        return _cache[sig], {}
    timings = {}
    best, best_ms = None, float("inf")
    for cand in candidates or DEFAULT_CANDIDATES:
        batch.prepare(Tuning(cand.ctaThreads, cand.tileLookups, cand.order, 0))
        batch.launch()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(reps):
            batch.launch()
        e.record()
        torch.cuda.synchronize(batch.device)
        ms = s.elapsed_time(e) / reps
        timings[cand.as_tuple()] = ms
        if ms < best_ms:
            best, best_ms = Tuning(cand.ctaThreads, cand.tileLookups, cand.order, 0), ms
    batch.prepare(best)
    _cache[sig] = best
    return best, timings
