"""The continuous-batching server: every request's shares are identical whether it ran alone
through the per-call C ABI or mixed into batched launches with others; admission respects
the key-store capacity; the plain mode serves the same arrivals."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def pools():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from fastfunctionsecretsharing_b200 import serving as S

    return S.make_pools("cuda", dcf_log2=(10, 14), spline_log2=(10, 11), seed=3)


@pytest.mark.parametrize("mode", ["batched", "plain"])
def test_alone_equals_mixed(pools, mode):
    from fastfunctionsecretsharing_b200 import serving as S

    reqs = S.make_requests(pools, rate=3000.0, count=48, seed=21, dcf_log2=(10, 14), spline_log2=(10, 11))
    # capacity for ~3 of the largest spline requests: admission must queue some requests
    cap = 3 * (1 << 11) * S.SPLINE_KEY_BYTES
    srv = S.Server(pools, capacity_bytes=cap, slots=3)
    makespan = srv.run(reqs, mode=mode)
    assert srv.store.peak <= cap and srv.store.used == 0
    alone = S.reference_outputs(srv, reqs)
    for r, a in zip(reqs, alone):
        assert np.array_equal(r.out_host.numpy(), a), (r.rid, r.kind, r.size)
    st = S.summarize(reqs, makespan)
    assert st["requests"] == 48 and st["p99_ms"] >= st["p50_ms"] > 0
    if mode == "batched":
        assert srv.launches < len(reqs)  # requests were batched together


def test_trace_shape():
    from fastfunctionsecretsharing_b200 import serving as S

    tr = S.mlp_trace(np.random.default_rng(0))
    per_layer = {}
    for kind, layer, size in tr:
        assert size & (size - 1) == 0
        per_layer[(kind, layer)] = per_layer.get((kind, layer), 0) + size
    assert len(per_layer) == 24 and set(per_layer.values()) == {1 << 18}
