"""DCF / DPF on the GPU through the C ABI (fastfunctionsecretsharing_b200 -> libFastFss.so):
bit-exact keys and shares against the golden fixtures (reference CPU outputs) and against
the oracle on seeded grids modelled on tests/dcf/dcf_eval_cuda.cu and tests/dpf/*."""

import zlib

import numpy as np
import pytest
from conftest import golden_names, load_golden
from fss_cases import DTYPES, rnd, seeds

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def F():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import fastfunctionsecretsharing_b200 as F

    return F


from gpu_util import dev_bytes, dev_ring, empty_bytes, empty_ring, host  # noqa: E402


def _dcf(F, kind, a, b, s0, s1, n, bo, g):
    es = a.dtype.itemsize
    key = empty_bytes()
    getattr(F, f"{kind}_key_gen")(key, dev_ring(a), dev_ring(b) if b is not None else empty_ring(es),
                                  dev_bytes(s0), dev_bytes(s1), n, bo, g)
    return key


def _eval(F, kind, key, x, s, p, n, bo, g):
    es = x.dtype.itemsize
    out = empty_ring(es)
    getattr(F, f"{kind}_eval")(out, dev_ring(x), key, dev_bytes(s), p, n, bo, g)
    return host(out, es)


@pytest.mark.parametrize("name", golden_names("dcf_u") + golden_names("dpf_u"))
def test_golden(F, name):
    g = load_golden(name)
    kind = name[:3]
    key = _dcf(F, kind, g["alpha"], g["beta"], g["seed0"], g["seed1"], g["n"], g["bo"], g["g"])
    assert np.array_equal(host(key), g["key"]), "key bytes differ from the reference"
    for p in (0, 1):
        y = _eval(F, kind, key, g["maskedX"], g[f"seed{p}"], p, g["n"], g["bo"], g["g"])
        assert np.array_equal(y, g[f"y{p}"]), f"party {p} shares differ from the reference"


WIDTHS = [(es, n, bo) for es in (1, 2, 4, 8) for n in sorted({1, 8 * es - 1, 8 * es})
          for bo in sorted({1, 8 * es - 1, 8 * es})]


@pytest.mark.parametrize("es,n,bo", WIDTHS)
@pytest.mark.parametrize("g", [1, 2, 3, 4])
@pytest.mark.parametrize("kind", ["dcf", "dpf"])
def test_grid_vs_oracle(F, oracle, kind, es, n, bo, g):
    rng = np.random.default_rng(zlib.crc32(repr((kind, es, n, bo, g)).encode()))
    N = 1023 if (es, g) == (4, 1) else 257
    a, b, s0, s1 = rnd(rng, N, es, n), rnd(rng, N * g, es, bo), seeds(rng, N), seeds(rng, N)
    x = rnd(rng, N, es, 8 * es)
    x[::5] = a[::5]
    kref = getattr(oracle, f"{kind}_keygen")(a, b, s0, s1, n, bo, g)
    key = _dcf(F, kind, a, b, s0, s1, n, bo, g)
    assert np.array_equal(host(key), kref)
    for p, s in ((0, s0), (1, s1)):
        want = getattr(oracle, f"{kind}_eval")(x, kref, s, p, n, bo, g)
        assert np.array_equal(_eval(F, kind, key, x, s, p, n, bo, g), want)


@pytest.mark.parametrize("N", [0, 1, 8, 1023, 1024, 2047, 2048])
@pytest.mark.parametrize("kind", ["dcf", "dpf"])
def test_element_counts(F, oracle, kind, N):
    rng = np.random.default_rng(N)
    es, n, bo, g = 4, 32, 32, 1
    a, b, s0, s1 = rnd(rng, N, es, n), rnd(rng, N, es, bo), seeds(rng, N), seeds(rng, N)
    x = rnd(rng, N, es, n)
    x[::7] = a[::7]
    key = _dcf(F, kind, a, b, s0, s1, n, bo, g)
    assert np.array_equal(host(key), getattr(oracle, f"{kind}_keygen")(a, b, s0, s1, n, bo, g))
    for p, s in ((0, s0), (1, s1)):
        want = getattr(oracle, f"{kind}_eval")(x, host(key), s, p, n, bo, g)
        assert np.array_equal(_eval(F, kind, key, x, s, p, n, bo, g), want)


def test_beta_default_is_one(F, oracle):
    rng = np.random.default_rng(5)
    es, n, bo, N = 2, 16, 16, 300
    a, s0, s1 = rnd(rng, N, es, n), seeds(rng, N), seeds(rng, N)
    for kind in ("dcf", "dpf"):
        key = _dcf(F, kind, a, None, s0, s1, n, bo, 1)
        assert np.array_equal(host(key), getattr(oracle, f"{kind}_keygen")(a, None, s0, s1, n, bo, 1))


def test_dpf_eval_all_and_multi_golden(F):
    g = load_golden("dpf_eval_all_u8_n6_g2")
    for p in (0, 1):
        out = empty_ring(1)
        F.dpf_eval_all(out, dev_ring(g["maskedX"]), dev_bytes(g["key"]), dev_bytes(g[f"seed{p}"]), p, g["n"], g["bo"],
                       g["g"])
        assert np.array_equal(host(out, 1), g[f"y{p}"])
    g = load_golden("dpf_eval_multi_u16_n10")
    for p in (0, 1):
        out = empty_ring(2)
        F.dpf_multi_eval(out, dev_ring(g["maskedX"]), dev_bytes(g["key"]), dev_bytes(g[f"seed{p}"]), p,
                         dev_ring(g["point"]), g["n"], g["bo"], g["g"])
        assert np.array_equal(host(out, 2), g[f"y{p}"])


@pytest.mark.parametrize("es,n,g", [(1, 8, 1), (2, 10, 3), (4, 12, 1), (8, 9, 2), (1, 1, 1), (1, 3, 2), (2, 6, 1),
                                    (4, 7, 1), (8, 5, 17), (4, 14, 1), (2, 16, 1)])
def test_dpf_eval_all_multi_vs_oracle(F, oracle, es, n, g):
    """Full domain: depth-first subtrees of up to 2^7 leaves under a walked prefix (n > 7), a
    single subtree per element (n <= 7); multi-value leaves through the AES-CTR convert (g = 17)."""
    rng = np.random.default_rng(es * 100 + n)
    N, bo = 9, 8 * es
    a, b, s0, s1 = rnd(rng, N, es, n), rnd(rng, N * g, es, bo), seeds(rng, N), seeds(rng, N)
    key = oracle.dpf_keygen(a, b, s0, s1, n, bo, g)
    x = rnd(rng, N, es, 8 * es)
    pt = rnd(rng, 17, es, 8 * es)
    for p, s in ((0, s0), (1, s1)):
        out = empty_ring(es)
        F.dpf_eval_all(out, dev_ring(x), dev_bytes(key), dev_bytes(s), p, n, bo, g)
        assert np.array_equal(host(out, es), oracle.dpf_eval_all(x, key, s, p, n, bo, g))
        out = empty_ring(es)
        F.dpf_multi_eval(out, dev_ring(x), dev_bytes(key), dev_bytes(s), p, dev_ring(pt), n, bo, g)
        assert np.array_equal(host(out, es), oracle.dpf_eval_multi(x, key, s, p, pt, n, bo, g))


def test_full_size_reconstruction_dcf_n32(F):
    """BASELINE config-2 size (2^24 elements, n = 32, Z_2^32): shares of both parties
    reconstruct beta * [maskedX < alpha] on every element (checked on the device)."""
    N, n = 1 << 24, 32
    gen = torch.Generator(device="cuda").manual_seed(7)
    a = torch.randint(-2**31, 2**31, (N,), dtype=torch.int32, device="cuda", generator=gen)
    b = torch.randint(-2**31, 2**31, (N,), dtype=torch.int32, device="cuda", generator=gen)
    s0 = torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device="cuda", generator=gen)
    s1 = torch.randint(0, 256, (N * 16,), dtype=torch.uint8, device="cuda", generator=gen)
    x = torch.randint(-2**31, 2**31, (N,), dtype=torch.int32, device="cuda", generator=gen)
    mx = x + a  # wraps mod 2^32
    key = torch.empty(0, dtype=torch.uint8, device="cuda")
    F.dcf_key_gen(key, a, b, s0, s1, n, n, 1)
    y0 = torch.empty(0, dtype=torch.int32, device="cuda")
    y1 = torch.empty(0, dtype=torch.int32, device="cuda")
    F.dcf_eval(y0, mx, key, s0, 0, n, n, 1)
    F.dcf_eval(y1, mx, key, s1, 1, n, n, 1)
    lt = (mx.to(torch.int64) & 0xFFFFFFFF) < (a.to(torch.int64) & 0xFFFFFFFF)
    want = torch.where(lt, b, torch.zeros_like(b))
    assert torch.equal((y0 + y1).view(-1), want)
    del key
    torch.cuda.empty_cache()


@pytest.mark.parametrize("es,n", [(4, 32), (8, 64), (2, 13), (1, 3)])
@pytest.mark.parametrize("kind", ["dcf", "dpf"])
def test_staged_eval_partial_tiles(F, oracle, kind, es, n):
    """groupSize-1 DCF and DPF evaluation stage correction words through shared memory, 32
    elements per warp and 4 levels per copy: element counts that leave partial warp tiles and
    widths that leave a partial last copy give the oracle's shares, no staging wait runs out,
    and a key that is not 16-byte aligned is refused before anything is launched."""
    import ctypes

    from fastfunctionsecretsharing_b200 import _lib

    rng = np.random.default_rng(zlib.crc32(repr(("staged", es, n)).encode()))
    for N in (1, 33, 4099):
        a, b, s0 = rnd(rng, N, es, n), rnd(rng, N, es, 8 * es), seeds(rng, N)
        s1 = seeds(rng, N)
        kref = getattr(oracle, f"{kind}_keygen")(a, b, s0, s1, n, 8 * es, 1)
        x = rnd(rng, N, es, 8 * es)
        x[::3] = a[::3]
        for p, s in ((0, s0), (1, s1)):
            out = empty_ring(es)
            getattr(F, f"{kind}_eval")(out, dev_ring(x), dev_bytes(kref), dev_bytes(s), p, n, 8 * es, 1)
            assert np.array_equal(host(out, es), getattr(oracle, f"{kind}_eval")(x, kref, s, p, n, 8 * es, 1))
    buf = torch.zeros(kref.size + 8, dtype=torch.uint8, device="cuda")
    unaligned = buf[8:]
    assert unaligned.data_ptr() % 16 == 8
    with pytest.raises(RuntimeError, match="failed : -1"):
        getattr(F, f"{kind}_eval")(empty_ring(es), dev_ring(x), unaligned, dev_bytes(s0), 0, n, 8 * es, 1)
    torch.cuda.synchronize()
    cnt = ctypes.c_uint(7)
    assert _lib.fn("FastFss_b200_stageTimeouts")(ctypes.byref(cnt)) == 0
    assert cnt.value == 0


def test_config1_keygen_eval_full_size(F, oracle):
    """The plain DCF keyGen + eval workload the reference's CPU path is timed on: 2^16 elements,
    n = 16, output Z_2^16 stored as uint16, seeded alpha, beta, mask m and 128-bit seeds,
    maskedX = (m + alpha) mod 2^16. GPU keys and both parties' shares equal the oracle's byte
    for byte, and the shares reconstruct beta * [maskedX < alpha] (the reference's test
    identity, tests/dcf/dcf_eval_test_case.h)."""
    rng = np.random.default_rng(20160)
    N, n, es = 1 << 16, 16, 2
    a, b, m = rnd(rng, N, es, n), rnd(rng, N, es, n), rnd(rng, N, es, n)
    s0, s1 = seeds(rng, N), seeds(rng, N)
    x = ((m.astype(np.uint32) + a.astype(np.uint32)) & 0xFFFF).astype(np.uint16)
    kref = oracle.dcf_keygen(a, b, s0, s1, n, n, 1)
    key = _dcf(F, "dcf", a, b, s0, s1, n, n, 1)
    assert np.array_equal(host(key), kref)
    y = []
    for p, s in ((0, s0), (1, s1)):
        got = _eval(F, "dcf", key, x, s, p, n, n, 1)
        assert np.array_equal(got, oracle.dcf_eval(x, kref, s, p, n, n, 1))
        y.append(got.astype(np.uint32))
    want = np.where(x.astype(np.uint32) < a.astype(np.uint32), b.astype(np.uint32), 0)
    assert np.array_equal((y[0] + y[1]) & 0xFFFF, want)
