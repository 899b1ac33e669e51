"""The batched persistent launch (include/FastFss/b200/batch.h): every request's output is
bit-identical to its per-call C-ABI result and to the oracle, directly, through a captured
CUDA graph, and under every autotuner candidate."""

import numpy as np
import pytest
from fss_cases import DTYPES, random_intervals, rnd, seeds, sorted_partition

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from gpu_util import dev_bytes, dev_ring, empty_ring, host  # noqa: E402


@pytest.fixture(scope="module")
def F():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import fastfunctionsecretsharing_b200 as F

    return F


def build_mixed(oracle, rng):
    """A small mixed batch: every kind, several widths, uneven sizes; returns (requests,
    expected outputs)."""
    from fastfunctionsecretsharing_b200 import batch as B

    reqs, want = [], []
    for kind, es, n, bo, N, extra in [
        ("dcf", 4, 32, 32, 3000, None), ("dcf", 1, 7, 8, 77, None), ("dcf", 8, 64, 64, 1, None),
        ("dpf", 2, 12, 16, 900, None), ("dpf", 8, 50, 64, 33, None),
        ("mic", 8, 64, 64, 200, 5), ("mic", 2, 12, 12, 515, 16), ("mic", 1, 8, 8, 64, 3),
        ("spline", 8, 64, 64, 37, (4, 2)), ("spline", 4, 24, 32, 100, (3, 1)), ("spline", 2, 16, 16, 9, (33, 0)),
        ("grotto", 2, 16, 16, 1000, True), ("grotto", 8, 64, 64, 50, False), ("grotto", 1, 6, 6, 40, True),
    ]:
        party = int(rng.integers(0, 2))
        a, s0, s1 = rnd(rng, N, es, n), seeds(rng, N), seeds(rng, N)
        s = s1 if party else s0
        x = rnd(rng, N, es, 8 * es)
        out = empty_ring(es)
        if kind == "dcf":
            k = oracle.dcf_keygen(a, rnd(rng, N, es, bo), s0, s1, n, bo, 1)
            reqs.append(B.dcf_request(out, dev_ring(x), dev_bytes(k), dev_bytes(s), party, n, bo))
            want.append(oracle.dcf_eval(x, k, s, party, n, bo, 1))
        elif kind == "dpf":
            k = oracle.dpf_keygen(a, rnd(rng, N, es, bo), s0, s1, n, bo, 1)
            reqs.append(B.dpf_request(out, dev_ring(x), dev_bytes(k), dev_bytes(s), party, n, bo))
            want.append(oracle.dpf_eval(x, k, s, party, n, bo, 1))
        elif kind == "mic":
            L, R = random_intervals(rng, extra, es, n)
            k, z = oracle.dcf_mic_keygen(a, s0, s1, L, R, n, bo)
            zs = rnd(rng, z.size, es, 8 * es)
            reqs.append(B.mic_request(out, dev_ring(x), dev_bytes(k), dev_ring(zs), dev_bytes(s), party, dev_ring(L),
                                      dev_ring(R), n, bo))
            want.append(oracle.dcf_mic_eval(x, k, zs, s, party, L, R, n, bo))
        elif kind == "spline":
            m, d = extra
            L, R = sorted_partition(rng, m, es, n)
            c = rnd(rng, m * (d + 1), es, 8 * es)
            k, e, beta = oracle.spline_keygen(a, s0, s1, c, d, L, R, n, bo)
            reqs.append(B.spline_request(out, dev_ring(x), dev_bytes(k), dev_ring(e), dev_ring(beta), dev_bytes(s),
                                         party, dev_ring(L), dev_ring(R), m, d, n, bo))
            want.append(oracle.spline_eval(x, k, e, beta, s, party, L, R, d, n, bo))
        else:
            k = oracle.grotto_keygen(a, s0, s1, n)
            reqs.append(B.grotto_request(out, dev_ring(x), dev_bytes(k), dev_bytes(s), extra, party, n))
            want.append(oracle.grotto_eval(x, k, s, extra, party, n))
    return reqs, want


def check(reqs, want):
    for r, w in zip(reqs, want):
        got = host(r.tensors[0], w.dtype.itemsize)
        assert np.array_equal(got, w), (r.op.kind, r.op.elementSize, r.op.bitWidthIn)


def test_mixed_batch_matches_oracle(F, oracle):
    from fastfunctionsecretsharing_b200 import batch as B

    reqs, want = build_mixed(oracle, np.random.default_rng(11))
    b = B.Batch(reqs).prepare()
    b.launch()
    torch.cuda.synchronize()
    check(reqs, want)
    # every launch shape yields the same shares
    for cand in B.DEFAULT_CANDIDATES:
        for r in reqs:
            r.tensors[0].zero_()
        b.prepare(cand)
        b.launch()
        torch.cuda.synchronize()
        check(reqs, want)


def test_graph_replay(F, oracle):
    from fastfunctionsecretsharing_b200 import batch as B

    reqs, want = build_mixed(oracle, np.random.default_rng(12))
    b = B.Batch(reqs).prepare(B.Tuning(256, 1 << 24, 0, 0))
    g = b.graph()
    for _ in range(3):
        for r in reqs:
            r.tensors[0].fill_(7)
        g.replay()
        torch.cuda.synchronize()
        check(reqs, want)


def test_autotune_and_config4_sample(F):
    """A scaled mixed-bitwidth MIC + spline sample: batched outputs equal the plain per-call
    C-ABI loop's, bit for bit; the autotuner returns one of its candidates."""
    from fastfunctionsecretsharing_b200 import batch as B
    from fastfunctionsecretsharing_b200 import workloads as W

    inst = W.mixed_mic_spline(instances=24, seed=5, mic_log2=(8, 12), spline_log2=(8, 9))
    W.run_plain(inst)
    b = B.Batch([i.request for i in inst])
    best, timings = B.autotune(b, reps=1)
    assert best.as_tuple() in timings
    b.launch()
    torch.cuda.synchronize()
    for i in inst:
        assert torch.equal(i.request.tensors[0].view(-1), i.out_plain.view(-1)), (i.kind, i.n, i.N)


def test_rejects_invalid(F):
    from fastfunctionsecretsharing_b200 import batch as B

    x = torch.zeros(4, dtype=torch.int32, device="cuda")
    key = torch.zeros(16, dtype=torch.uint8, device="cuda")
    r = B.dcf_request(torch.empty(0, dtype=torch.int32, device="cuda"), x, key, key, 2, 32, 32)
    with pytest.raises(RuntimeError, match=": -12"):
        B.Batch([r]).prepare()
    r = B.dcf_request(torch.empty(0, dtype=torch.int32, device="cuda"), x, key, key, 0, 33, 32)
    with pytest.raises(RuntimeError, match=": -10"):
        B.Batch([r]).prepare()
