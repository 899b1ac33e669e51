"""Multi-rank element sharding without a GPU: ranges partition the batch, per-rank key slices
are exactly the keys of the sub-batch, and two gloo ranks that each evaluate their shard
(with the CPU oracle standing in for the device) reproduce the single-rank shares; the
max-over-ranks timing reduction works over the process group."""

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp
from fss_cases import dcf_regions, rnd, seeds

from fastfunctionsecretsharing_b200.sharding import key_slice_offsets, max_over_ranks, shard_range


@pytest.mark.parametrize("n", [0, 1, 7, 1000, 1 << 20])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_range_partitions(n, world):
    spans = [shard_range(n, r, world) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == n
    for (a, b), (c, d) in zip(spans, spans[1:]):
        assert b == c and a <= b
    sizes = [b - a for a, b in spans]
    assert max(sizes) - min(sizes) <= 1


def test_bad_rank():
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def sub_key(key, regions, N, begin, end):
    return np.concatenate([key[o:o + ln] for o, ln in key_slice_offsets(N, regions, begin, end)])


def test_key_slices_are_sub_batch_keys(oracle):
    rng = np.random.default_rng(3)
    es, n, bo, g, N = 4, 20, 32, 2, 101
    a, b, s0, s1 = rnd(rng, N, es, n), rnd(rng, N * g, es, bo), seeds(rng, N), seeds(rng, N)
    key = oracle.dcf_keygen(a, b, s0, s1, n, bo, g)
    for r in range(3):
        lo, hi = shard_range(N, r, 3)
        want = oracle.dcf_keygen(a[lo:hi], b[lo * g:hi * g], s0[16 * lo:16 * hi], s1[16 * lo:16 * hi], n, bo, g)
        assert np.array_equal(sub_key(key, dcf_regions(n, g, es), N, lo, hi), want)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle.pyoracle import Oracle

        O = Oracle()
        rng = np.random.default_rng(11)
        es, n, bo, N = 4, 32, 32, 64
        a, b, s0, s1 = rnd(rng, N, es, n), rnd(rng, N, es, bo), seeds(rng, N), seeds(rng, N)
        x = rnd(rng, N, es, n)
        key = O.dcf_keygen(a, b, s0, s1, n, bo, 1)
        lo, hi = shard_range(N, rank, world)
        k = sub_key(key, dcf_regions(n, 1, es), N, lo, hi)
        y = O.dcf_eval(x[lo:hi], k, s0[16 * lo:16 * hi], 0, n, bo, 1)
        t = max_over_ranks(float(rank + 1) * 1.5, world)
        q.put((rank, lo, hi, y.tobytes(), t))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_single_rank(oracle):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rng = np.random.default_rng(11)
    es, n, bo, N = 4, 32, 32, 64
    a, b, s0, s1 = rnd(rng, N, es, n), rnd(rng, N, es, bo), seeds(rng, N), seeds(rng, N)
    x = rnd(rng, N, es, n)
    full = oracle.dcf_eval(x, oracle.dcf_keygen(a, b, s0, s1, n, bo, 1), s0, 0, n, bo, 1)
    got = np.zeros(N, np.uint32)
    for rank, lo, hi, yb, t in res:
        got[lo:hi] = np.frombuffer(yb, np.uint32)
        assert t == 3.0  # max over ranks of (rank + 1) * 1.5
    assert np.array_equal(got, full)
