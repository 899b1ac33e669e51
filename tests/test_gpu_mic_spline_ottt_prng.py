"""DCF-MIC, spline, OTTT and the AES-CTR generator on the GPU through the C ABI, bit-exact
against the reference fixtures and the oracle (tests/mic, tests/spline, tests/ottt shapes)."""

import zlib

import numpy as np
import pytest
from conftest import golden_names, load_golden
from fss_cases import DTYPES, random_intervals, rnd, seeds, sorted_partition, touching_intervals

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from gpu_util import dev_bytes, dev_ring, empty_bytes, empty_ring, host  # noqa: E402


@pytest.fixture(scope="module")
def F():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import fastfunctionsecretsharing_b200 as F

    return F


def sub(a, b):
    return (a.astype(np.uint64) - b.astype(np.uint64)).astype(a.dtype)


@pytest.mark.parametrize("name", golden_names("dcf_mic_u"))
def test_mic_golden(F, name):
    g = load_golden(name)
    es = g["es"]
    key, z = empty_bytes(), empty_ring(es)
    F.dcf_mic_key_gen(key, z, dev_ring(g["alpha"]), dev_bytes(g["seed0"]), dev_bytes(g["seed1"]), dev_ring(g["left"]),
                      dev_ring(g["right"]), g["n"], g["bo"])
    assert np.array_equal(host(key), g["key"]) and np.array_equal(host(z, es), g["z"])
    for p in (0, 1):
        out = empty_ring(es)
        F.dcf_mic_eval(out, dev_ring(g["maskedX"]), key, dev_ring(g[f"z{p}"]), dev_bytes(g[f"seed{p}"]), p,
                       dev_ring(g["left"]), dev_ring(g["right"]), g["n"], g["bo"])
        assert np.array_equal(host(out, es), g[f"y{p}"])


@pytest.mark.parametrize("es,n,bo,m", [(1, 8, 8, 3), (2, 15, 16, 9), (4, 32, 32, 16), (8, 64, 64, 16), (8, 40, 17, 5),
                                       (4, 20, 32, 40), (2, 16, 16, 1)])
@pytest.mark.parametrize("layout", ["random", "touching", "tiling"])
def test_mic_vs_oracle(F, oracle, es, n, bo, m, layout):
    """Touching intervals (each point walked once and shared by the two intervals around it;
    tiling: the last also touches the first) and independent intervals (two walks per
    interval) give the oracle's shares."""
    rng = np.random.default_rng(zlib.crc32(repr(("dmic", es, n, bo, m, layout)).encode()))
    N = 257
    a, s0, s1 = rnd(rng, N, es, n), seeds(rng, N), seeds(rng, N)
    if layout == "random":
        L, R = random_intervals(rng, m, es, n)
    elif layout == "touching":
        L, R = touching_intervals(rng, m, es, n)
    else:
        L, R = sorted_partition(rng, m, es, n)
    kref, zref = oracle.dcf_mic_keygen(a, s0, s1, L, R, n, bo)
    key, z = empty_bytes(), empty_ring(es)
    F.dcf_mic_key_gen(key, z, dev_ring(a), dev_bytes(s0), dev_bytes(s1), dev_ring(L), dev_ring(R), n, bo)
    assert np.array_equal(host(key), kref) and np.array_equal(host(z, es), zref)
    z0 = rnd(rng, N * m, es, 8 * es)
    x = rnd(rng, N, es, 8 * es)
    for p, zs, s in ((0, z0, s0), (1, sub(zref, z0), s1)):
        out = empty_ring(es)
        F.dcf_mic_eval(out, dev_ring(x), key, dev_ring(zs), dev_bytes(s), p, dev_ring(L), dev_ring(R), n, bo)
        assert np.array_equal(host(out, es), oracle.dcf_mic_eval(x, kref, zs, s, p, L, R, n, bo))


@pytest.mark.parametrize("name", golden_names("spline_u"))
def test_spline_golden(F, name):
    g = load_golden(name)
    es, d, m = g["es"], g["d"], g["left"].size
    key, e, beta = empty_bytes(), empty_ring(es), empty_ring(es)
    F.spline_key_gen(key, e, beta, dev_ring(g["alpha"]), dev_bytes(g["seed0"]), dev_bytes(g["seed1"]),
                     dev_ring(g["coeffs"]), d, dev_ring(g["left"]), dev_ring(g["right"]), m, g["n"], g["bo"])
    assert np.array_equal(host(key), g["key"])
    assert np.array_equal(host(e, es), g["e"]) and np.array_equal(host(beta, es), g["beta"])
    for p in (0, 1):
        out = empty_ring(es)
        F.spline_eval(out, dev_ring(g["maskedX"]), key, dev_ring(g[f"e{p}"]), dev_ring(g[f"b{p}"]),
                      dev_bytes(g[f"seed{p}"]), p, dev_ring(g["left"]), dev_ring(g["right"]), m, d, g["n"], g["bo"])
        assert np.array_equal(host(out, es), g[f"y{p}"])


@pytest.mark.parametrize("es,n,bo,m,d", [(8, 64, 64, 32, 2), (2, 16, 16, 7, 1), (4, 32, 24, 4, 5), (1, 8, 8, 3, 0),
                                         (8, 48, 64, 2, 8), (8, 40, 40, 5, 1), (8, 64, 56, 3, 3), (4, 32, 32, 2, 0),
                                         (2, 12, 12, 5, 2), (4, 32, 32, 9, 2), (8, 64, 64, 1, 0)])
@pytest.mark.parametrize("layout", ["partition", "rotated", "gaps"])
def test_spline_vs_oracle(F, oracle, es, n, bo, m, d, layout):
    """Intervals that tile the ring (a partition from 0, or one rotated so that an interval
    wraps) take the shared-endpoint walks; intervals with gaps take one walk per endpoint."""
    rng = np.random.default_rng(zlib.crc32(repr(("spline", es, n, bo, m, d, layout)).encode()))
    N = 40
    a, s0, s1 = rnd(rng, N, es, n), seeds(rng, N), seeds(rng, N)
    if layout == "gaps":
        L, R = random_intervals(rng, m, es, n)
    else:
        L, R = sorted_partition(rng, m, es, n)
        if layout == "rotated":
            r = int(rnd(rng, 1, 8, n)[0])
            mask = (1 << n) - 1
            L = np.array([(int(v) + r) & mask for v in L], dtype=np.uint64).astype(L.dtype)
            R = np.array([(int(v) + r) & mask for v in R], dtype=np.uint64).astype(R.dtype)
    c = rnd(rng, m * (d + 1), es, 8 * es)
    kref, eref, bref = oracle.spline_keygen(a, s0, s1, c, d, L, R, n, bo)
    key, e, beta = empty_bytes(), empty_ring(es), empty_ring(es)
    F.spline_key_gen(key, e, beta, dev_ring(a), dev_bytes(s0), dev_bytes(s1), dev_ring(c), d, dev_ring(L), dev_ring(R),
                     m, n, bo)
    assert np.array_equal(host(key), kref)
    assert np.array_equal(host(e, es), eref) and np.array_equal(host(beta, es), bref)
    e0, b0 = rnd(rng, eref.size, es, 8 * es), rnd(rng, bref.size, es, 8 * es)
    x = rnd(rng, N, es, 8 * es)
    for p, es_, bs, s in ((0, e0, b0, s0), (1, sub(eref, e0), sub(bref, b0), s1)):
        out = empty_ring(es)
        F.spline_eval(out, dev_ring(x), key, dev_ring(es_), dev_ring(bs), dev_bytes(s), p, dev_ring(L), dev_ring(R), m, d,
                      n, bo)
        assert np.array_equal(host(out, es), oracle.spline_eval(x, kref, es_, bs, s, p, L, R, d, n, bo))


@pytest.mark.parametrize("name", golden_names("ottt_u"))
def test_ottt_golden(F, name):
    g = load_golden(name)
    es = g["es"]
    k = dev_bytes(g["key0"])
    F.ottt_key_gen(k, dev_ring(g["alpha"]), g["n"])
    assert np.array_equal(host(k), g["key1"])
    for p in (0, 1):
        oe, ot = empty_ring(es), empty_ring(es)
        F.ottt_lut_eval(oe, ot, dev_ring(g["maskedX"]), dev_bytes(g[f"key{p}"]), p, dev_ring(g["lut"]), g["n"], 8 * es)
        assert np.array_equal(host(oe, es), g[f"e{p}"]) and np.array_equal(host(ot, es), g[f"t{p}"])


@pytest.mark.parametrize("es,n,lutn", [(1, 3, 1), (1, 4, 2), (2, 9, 5), (4, 12, 1), (8, 6, 9), (2, 16, 1)])
def test_ottt_vs_oracle(F, oracle, es, n, lutn):
    rng = np.random.default_rng(es * 100 + n)
    N = 77
    a = rnd(rng, N, es, 8 * es)
    k0 = rng.integers(0, 256, size=N * (1 << n) // 8, dtype=np.uint8)
    lut = rnd(rng, (1 << n) * lutn, es, 8 * es)
    x = rnd(rng, N, es, 8 * es)
    k = dev_bytes(k0)
    F.ottt_key_gen(k, dev_ring(a), n)
    k1 = oracle.ottt_keygen(k0, a, n)
    assert np.array_equal(host(k), k1)
    for p, kk in ((0, k0), (1, k1)):
        oe, ot = empty_ring(es), empty_ring(es)
        F.ottt_lut_eval(oe, ot, dev_ring(x), dev_bytes(kk), p, dev_ring(lut), n, 8 * es)
        we, wt = oracle.ottt_lut_eval(x, kk, p, lut, n)
        assert np.array_equal(host(oe, es), we) and np.array_equal(host(ot, es), wt)


def test_prng_golden_and_counter(F, oracle):
    g = load_golden("prng")
    P = F.Prng("cuda")
    P.set_current_seed(g["seed"].tobytes(), g["counter"].tobytes())
    out = torch.empty(g["out"].size, dtype=torch.uint8, device="cuda")
    assert P.rand_(out, 8) is out
    assert np.array_equal(host(out), g["out"])
    assert P.get_current_seed()[1] == g["counter_after"].tobytes()
    # a second call continues the stream exactly like the CPU generator
    out2 = torch.empty(333, dtype=torch.uint8, device="cuda")
    P.rand_(out2, 8)
    want, ctr = oracle.prng(g["seed"].tobytes(), g["counter_after"].tobytes(), 333)
    assert np.array_equal(host(out2), want) and P.get_current_seed()[1] == ctr
    # unaligned destination
    buf = torch.zeros(1000, dtype=torch.uint8, device="cuda")
    P.set_current_seed(bytes(16), bytes(16))
    P.rand_(buf[3:3 + 500], 8)
    want, _ = oracle.prng(bytes(16), bytes(16), 500)
    assert np.array_equal(host(buf[3:503]), want) and not host(buf[:3]).any()
    # the reference binding's contract: 16-byte seed and counter, device() and to_()
    assert P.device() == torch.device("cuda")
    with pytest.raises(RuntimeError, match="16 bytes"):
        P.set_current_seed(bytes(8), bytes(16))
    before = P.get_current_seed()
    assert P.to_(torch.device("cuda", 0)) is P and P.get_current_seed() == before
