"""FastFss_cuda_batchEvalNoAlloc: the batched evaluation for callers that cannot allocate device
memory (its queue and descriptor table live in a fixed array inside the library). Called
through the C ABI twice in a row — with two different batches, so the second call runs on the
array the first one left behind — each result must equal, bit for bit, what the workspace-based
entry points (FastFss_cuda_batchPrepare + FastFss_cuda_batchLaunch) produce for the same batch.
This module is collected last, and builds everything it needs itself, so it runs the same alone
in a fresh process or after the rest of the suite."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from fastfunctionsecretsharing_b200 import _lib

    f = _lib.fn("FastFss_cuda_batchEvalNoAlloc")
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p]
    return f


def make_batch(seed, counts):
    """Requests of every kind (DCF, DPF, MIC, spline, Grotto) over several widths; keys come
    from this library's own key generation."""
    import fastfunctionsecretsharing_b200 as F
    from fastfunctionsecretsharing_b200 import batch as B
    from fastfunctionsecretsharing_b200.workloads import TORCH_DT, _rand_ring, _ring_tensor, partition

    dev = torch.device("cuda")
    gen = torch.Generator(device=dev).manual_seed(seed)
    rng = np.random.default_rng(seed)
    reqs = []

    def seeds(N):
        return (torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device=dev, generator=gen),
                torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device=dev, generator=gen))

    for q, N in enumerate(counts):
        kind = q % 5
        es, n = [(4, 32), (2, 16), (8, 64), (1, 8)][q % 4]
        a = _rand_ring(gen, (N,), es, dev)
        x = _rand_ring(gen, (N,), es, dev)
        s0, s1 = seeds(N)
        out = torch.empty(0, dtype=TORCH_DT[es], device=dev)
        key = torch.empty(0, dtype=torch.uint8, device=dev)
        if kind == 0:
            F.dcf_key_gen(key, a, _rand_ring(gen, (N,), es, dev), s0, s1, n, n, 1)
            reqs.append(B.dcf_request(out, x, key, s0, 0, n, n))
        elif kind == 1:
            F.dpf_key_gen(key, a, _rand_ring(gen, (N,), es, dev), s0, s1, n, n, 1)
            reqs.append(B.dpf_request(out, x, key, s1, 1, n, n))
        elif kind == 2:
            L, R = partition(rng, 6, n)
            Lt, Rt = _ring_tensor(L, es, dev), _ring_tensor(R, es, dev)
            z = torch.empty(0, dtype=TORCH_DT[es], device=dev)
            F.dcf_mic_key_gen(key, z, a, s0, s1, Lt, Rt, n, n)
            reqs.append(B.mic_request(out, x, key, z, s0, 0, Lt, Rt, n, n))
        elif kind == 3:
            m, d = 4, 2
            L, R = partition(rng, m, n)
            Lt, Rt = _ring_tensor(L, es, dev), _ring_tensor(R, es, dev)
            c = _ring_tensor([int(v) for v in rng.integers(0, 2**62, size=m * (d + 1))], es, dev)
            e = torch.empty(0, dtype=TORCH_DT[es], device=dev)
            beta = torch.empty(0, dtype=TORCH_DT[es], device=dev)
            F.spline_key_gen(key, e, beta, a, s0, s1, c, d, Lt, Rt, m, n, n)
            reqs.append(B.spline_request(out, x, key, e, beta, s1, 1, Lt, Rt, m, d, n, n))
        else:
            F.grotto_key_gen(key, a, s0, s1, n)
            reqs.append(B.grotto_request(out, x, key, s0, True, 0, n))
    torch.cuda.synchronize()
    return reqs


def run_workspace(reqs):
    from fastfunctionsecretsharing_b200 import batch as B

    B.Batch(reqs).prepare().launch()
    torch.cuda.synchronize()
    return [r.tensors[0].clone() for r in reqs]


def run_no_alloc(lib, reqs):
    from fastfunctionsecretsharing_b200 import batch as B

    for r in reqs:
        r.tensors[0].fill_(0x5A)
    ops = (B.BatchOp * len(reqs))(*[r.op for r in reqs])
    tuning = B.Tuning(256, 1 << 24, 0, 0)
    h = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib(ctypes.addressof(ops), len(reqs), ctypes.addressof(tuning), ctypes.addressof(h))
    assert rc == 0, rc
    torch.cuda.synchronize()
    return [r.tensors[0].clone() for r in reqs]


def test_no_alloc_matches_workspace_entry_two_calls(lib):
    first = make_batch(31, [700, 515, 64, 40, 300, 129, 1, 2048, 33, 90])
    second = make_batch(32, [17, 1000, 260])
    for reqs in (first, second):
        want = run_workspace(reqs)
        got = run_no_alloc(lib, reqs)
        for w, g, r in zip(want, got, reqs):
            assert torch.equal(w, g), (r.op.kind, r.op.elementSize, r.op.elementNum)


def test_no_alloc_rejects_too_many_ops(lib):
    from fastfunctionsecretsharing_b200 import batch as B

    cap = 512
    ops = (B.BatchOp * (cap + 1))()
    h = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib(ctypes.addressof(ops), cap + 1, None, ctypes.addressof(h)) == -32
