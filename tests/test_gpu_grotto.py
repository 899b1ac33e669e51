"""Grotto on the GPU through the C ABI: keys and eq / lt / le / MIC / interval-LUT shares
bit-exact against the reference fixtures and the oracle; full-domain rows against the
reference's per-point evaluations (tests/grotto/*.cpp shapes; BASELINE config 3 at n = 16)."""

import zlib

import numpy as np
import pytest
from conftest import golden_names, load_golden
from fss_cases import random_intervals, rnd, seeds, sorted_partition, touching_intervals

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from gpu_util import dev_bytes, dev_ring, empty_bytes, empty_ring, host  # noqa: E402


@pytest.fixture(scope="module")
def F():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import fastfunctionsecretsharing_b200 as F

    return F


def keygen(F, a, s0, s1, n):
    key = empty_bytes()
    F.grotto_key_gen(key, dev_ring(a), dev_bytes(s0), dev_bytes(s1), n)
    return key


def point(F, op, x, key, s, p, n, eb=None):
    es = x.dtype.itemsize
    out = empty_ring(es)
    if op == "eq":
        F.grotto_eq_eval(out, dev_ring(x), key, dev_bytes(s), p, n)
    else:
        F.grotto_eval(out, dev_ring(x), key, dev_bytes(s), eb, p, n)
    return host(out, es)


@pytest.mark.parametrize("name", golden_names("grotto_u"))
def test_golden(F, name):
    g = load_golden(name)
    n, es = g["n"], g["es"]
    key = keygen(F, g["alpha"], g["seed0"], g["seed1"], n)
    assert np.array_equal(host(key), g["key"])
    for p in (0, 1):
        s = g[f"seed{p}"]
        assert np.array_equal(point(F, "eq", g["maskedX"], key, s, p, n), g[f"eq{p}"])
        assert np.array_equal(point(F, "cmp", g["maskedX"], key, s, p, n, False), g[f"lt{p}"])
        assert np.array_equal(point(F, "cmp", g["maskedX"], key, s, p, n, True), g[f"le{p}"])
        out = empty_ring(es)
        F.grotto_mic_eval(out, dev_ring(g["maskedX"]), key, dev_bytes(s), p, dev_ring(g["left"]), dev_ring(g["right"]), n)
        assert np.array_equal(host(out, es), g[f"mic{p}"])
        oe, ot = empty_ring(es), empty_ring(es)
        F.grotto_interval_lut_eval(oe, ot, dev_ring(g["maskedX"]), key, dev_bytes(s), p, dev_ring(g["left"]),
                                   dev_ring(g["right"]), dev_ring(g["lut"]), n, 8 * es)
        assert np.array_equal(host(oe, es), g[f"lutE{p}"]) and np.array_equal(host(ot, es), g[f"lutT{p}"])


GRID = [(es, n) for es in (1, 2, 4, 8) for n in sorted({6, 7, 8 * es - 1, 8 * es}) if 6 <= n <= 8 * es]


@pytest.mark.parametrize("es,n", GRID)
def test_grid_vs_oracle(F, oracle, es, n):
    rng = np.random.default_rng(zlib.crc32(repr(("grotto", es, n)).encode()))
    N = 517
    a, s0, s1 = rnd(rng, N, es, n), seeds(rng, N), seeds(rng, N)
    x = rnd(rng, N, es, 8 * es)
    x[::3] = a[::3]
    x[1::7] = 0
    kref = oracle.grotto_keygen(a, s0, s1, n)
    key = keygen(F, a, s0, s1, n)
    assert np.array_equal(host(key), kref)
    for p, s in ((0, s0), (1, s1)):
        assert np.array_equal(point(F, "eq", x, key, s, p, n), oracle.grotto_eq_eval(x, kref, s, p, n))
        for eb in (False, True):
            assert np.array_equal(point(F, "cmp", x, key, s, p, n, eb), oracle.grotto_eval(x, kref, s, eb, p, n))


@pytest.mark.parametrize("es,n,m,lutn", [(2, 16, 64, 1), (1, 8, 5, 3), (4, 20, 33, 6), (8, 64, 7, 2), (2, 12, 1, 2),
                                        (4, 24, 300, 9)])
@pytest.mark.parametrize("layout", ["partition", "touching", "random"])
def test_mic_lut_vs_oracle(F, oracle, es, n, m, lutn, layout):
    """Partitions (touching, the last round to the first), touching chains and independent
    intervals: each endpoint point walked once where intervals share it."""
    rng = np.random.default_rng(zlib.crc32(repr(("mic", es, n, m, layout)).encode()))
    N = 300
    a, s0, s1 = rnd(rng, N, es, n), seeds(rng, N), seeds(rng, N)
    kref = oracle.grotto_keygen(a, s0, s1, n)
    key = dev_bytes(kref)
    x = rnd(rng, N, es, 8 * es)
    if layout == "partition":
        L, R = sorted_partition(rng, m, es, n)
    elif layout == "touching":
        L, R = touching_intervals(rng, m, es, n)
    else:
        L, R = random_intervals(rng, m, es, n)
    lut = rnd(rng, m * lutn, es, 8 * es)
    for p, s in ((0, s0), (1, s1)):
        out = empty_ring(es)
        F.grotto_mic_eval(out, dev_ring(x), key, dev_bytes(s), p, dev_ring(L), dev_ring(R), n)
        assert np.array_equal(host(out, es), oracle.grotto_mic_eval(x, kref, s, p, L, R, n))
        oe, ot = empty_ring(es), empty_ring(es)
        F.grotto_interval_lut_eval(oe, ot, dev_ring(x), key, dev_bytes(s), p, dev_ring(L), dev_ring(R),
                                   dev_ring(lut), n, 8 * es)
        we, wt = oracle.grotto_interval_lut_eval(x, kref, s, p, L, R, lut, n, 8 * es)
        assert np.array_equal(host(oe, es), we) and np.array_equal(host(ot, es), wt)


def test_full_domain_golden(F):
    g = load_golden("grotto_all_u16_n10")
    N = g["alpha"].size
    for p in (0, 1):
        for op, k in ((F.grotto_eq_eval_all, "eqbits"), (F.grotto_le_eval_all, "lebits")):
            out = empty_bytes()
            op(out, dev_bytes(g["key"]), dev_bytes(g[f"seed{p}"]), p, g["n"], g["es"], N)
            assert np.array_equal(host(out), g[f"{k}{p}"])


@pytest.mark.parametrize("es,n", [(1, 6), (1, 8), (2, 11), (2, 16), (4, 12), (8, 17)])
def test_full_domain_vs_oracle(F, oracle, es, n):
    rng = np.random.default_rng(n * 10 + es)
    N = 6
    a, s0, s1 = rnd(rng, N, es, n), seeds(rng, N), seeds(rng, N)
    kref = oracle.grotto_keygen(a, s0, s1, n)
    for p, s in ((0, s0), (1, s1)):
        eq, le = empty_bytes(), empty_bytes()
        F.grotto_eq_eval_all(eq, dev_bytes(kref), dev_bytes(s), p, n, es, N)
        F.grotto_le_eval_all(le, dev_bytes(kref), dev_bytes(s), p, n, es, N)
        assert np.array_equal(host(eq), oracle.grotto_eq_eval_all(kref, s, p, n, es, N))
        assert np.array_equal(host(le), oracle.grotto_le_eval_all(kref, s, p, n, es, N))


@pytest.mark.parametrize("n", [7, 13])
def test_full_domain_rows_at_8_byte_offset(F, oracle, n):
    """Rows written to a buffer that is 8- but not 16-byte aligned (word-by-word stores) equal
    the oracle's, as do rows in an aligned buffer (paired 16-byte stores)."""
    rng = np.random.default_rng(n)
    N, es = 5, 2
    a, s0, s1 = rnd(rng, N, es, n), seeds(rng, N), seeds(rng, N)
    kref = oracle.grotto_keygen(a, s0, s1, n)
    nbytes = N * (1 << n) // 8
    for op, ref in ((F.grotto_eq_eval_all, oracle.grotto_eq_eval_all), (F.grotto_le_eval_all, oracle.grotto_le_eval_all)):
        buf = torch.zeros(nbytes + 16, dtype=torch.uint8, device="cuda")
        view = buf[8:8 + nbytes]
        assert view.data_ptr() % 16 == 8
        op(view, dev_bytes(kref), dev_bytes(s1), 1, n, es, N)
        assert np.array_equal(host(view), ref(kref, s1, 1, n, es, N))
        assert not host(buf[:8]).any() and not host(buf[8 + nbytes:]).any()


def test_full_domain_config3_reconstruction(F):
    """BASELINE config 3 size: 2^16 keys at n = 16, full domain. Party rows XOR to the one-hot
    of alpha (eq) and to the prefix [x <= alpha] (le) for every key (checked on the device)."""
    N, n = 1 << 16, 16
    gen = torch.Generator(device="cuda").manual_seed(3)
    a = torch.randint(0, 1 << 16, (N,), dtype=torch.int32, device="cuda", generator=gen).to(torch.int16)
    s0 = torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device="cuda", generator=gen)
    s1 = torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device="cuda", generator=gen)
    key = torch.empty(0, dtype=torch.uint8, device="cuda")
    F.grotto_key_gen(key, a, s0, s1, n)
    rows = []
    for op in (F.grotto_eq_eval_all, F.grotto_le_eval_all):
        r0, r1 = torch.empty(0, dtype=torch.uint8, device="cuda"), torch.empty(0, dtype=torch.uint8, device="cuda")
        op(r0, key, s0, 0, n, 2, N)
        op(r1, key, s1, 1, n, 2, N)
        rows.append((r0 ^ r1).view(N, -1))
    av = a.to(torch.int64) & 0xFFFF
    eq = rows[0]
    # exactly one set bit per row, at alpha
    pop = torch.zeros(N, dtype=torch.int64, device="cuda")
    for b in range(8):
        pop += ((eq >> b) & 1).sum(dim=1)
    assert torch.all(pop == 1)
    byte = eq.gather(1, (av // 8).view(-1, 1)).view(-1).to(torch.int64)
    assert torch.all((byte >> (av % 8)) & 1 == 1)
    le = rows[1].to(torch.int64)
    cnt = torch.zeros(N, dtype=torch.int64, device="cuda")
    for b in range(8):
        cnt += ((le >> b) & 1).sum(dim=1)
    assert torch.equal(cnt, av + 1)


@pytest.mark.parametrize("es,n,m,lutn", [(2, 16, 64, 1), (2, 10, 5, 6), (4, 20, 40, 2), (1, 8, 3, 1)])
def test_lut_from_rows_equals_walks(F, oracle, es, n, m, lutn):
    """The prefix-parity path (full-domain rows, then the LUT from rows) gives the shares of
    the walk-based interval LUT, which are the reference's."""
    rng = np.random.default_rng(n * 7 + m)
    N = 200
    a, s0, s1 = rnd(rng, N, es, n), seeds(rng, N), seeds(rng, N)
    kref = oracle.grotto_keygen(a, s0, s1, n)
    x = rnd(rng, N, es, 8 * es)
    L, R = sorted_partition(rng, m, es, n)
    lut = rnd(rng, m * lutn, es, 8 * es)
    for p, s in ((0, s0), (1, s1)):
        rows = empty_bytes()
        F.grotto_le_eval_all(rows, dev_bytes(kref), dev_bytes(s), p, n, es, N)
        oe, ot = empty_ring(es), empty_ring(es)
        F.grotto_interval_lut_eval_from_rows(oe, ot, dev_ring(x), rows, p, dev_ring(L), dev_ring(R), dev_ring(lut), n)
        we, wt = oracle.grotto_interval_lut_eval(x, kref, s, p, L, R, lut, n, 8 * es)
        assert np.array_equal(host(oe, es), we) and np.array_equal(host(ot, es), wt)
