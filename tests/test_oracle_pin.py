"""Pins the oracle restatement (oracle/fss_oracle.c) before anything is checked against it:
FIPS-197 known answers, every golden fixture produced by the reference's own CPU code, the
reconstruction identities of the reference's tests, and (when oracle/_ref is built) fresh
random cases against the reference library itself."""

import numpy as np
import pytest
from conftest import golden_names, load_golden
from fss_cases import DTYPES, random_intervals, rnd, seeds, sorted_partition


def test_aes_fips197_known_answer(oracle):
    # FIPS-197 Appendix C.1 (AES-128) and Appendix B.
    assert oracle.aes128(bytes(range(16)), bytes.fromhex("00112233445566778899aabbccddeeff")).hex() == \
        "69c4e0d86a7b0430d8cdb78070b4c55a"
    assert oracle.aes128(bytes.fromhex("2b7e151628aed2a6abf7158809cf4f3c"),
                         bytes.fromhex("3243f6a8885a308d313198a2e0370734")).hex() == "3925841d02dc09fbdc118597196a0b32"


def test_prng_golden(oracle):
    g = load_golden("prng")
    out, ctr = oracle.prng(g["seed"].tobytes(), g["counter"].tobytes(), g["out"].size)
    assert np.array_equal(out, g["out"])
    assert ctr == g["counter_after"].tobytes()


@pytest.mark.parametrize("name", golden_names("dcf_u"))
def test_dcf_golden(oracle, name):
    g = load_golden(name)
    key = oracle.dcf_keygen(g["alpha"], g["beta"], g["seed0"], g["seed1"], g["n"], g["bo"], g["g"])
    assert np.array_equal(key, g["key"])
    assert np.array_equal(oracle.dcf_eval(g["maskedX"], key, g["seed0"], 0, g["n"], g["bo"], g["g"]), g["y0"])
    assert np.array_equal(oracle.dcf_eval(g["maskedX"], key, g["seed1"], 1, g["n"], g["bo"], g["g"]), g["y1"])
    # tests/dcf/dcf_eval_test_case.h:73-86: y = beta * [maskedX < alpha] (mod 2^bo)
    bo, gs = g["bo"], g["g"]
    mo = (1 << bo) - 1
    y = (g["y0"].astype(object) + g["y1"].astype(object)) & mo
    exp = np.where(np.repeat(g["maskedX"].astype(object), gs) < np.repeat(g["alpha"].astype(object), gs),
                   g["beta"].astype(object), 0)
    assert all(int(a) == int(b) & mo for a, b in zip(y, exp))


@pytest.mark.parametrize("name", golden_names("dpf_u"))
def test_dpf_golden(oracle, name):
    g = load_golden(name)
    key = oracle.dpf_keygen(g["alpha"], g["beta"], g["seed0"], g["seed1"], g["n"], g["bo"], g["g"])
    assert np.array_equal(key, g["key"])
    y0 = oracle.dpf_eval(g["maskedX"], key, g["seed0"], 0, g["n"], g["bo"], g["g"])
    y1 = oracle.dpf_eval(g["maskedX"], key, g["seed1"], 1, g["n"], g["bo"], g["g"])
    assert np.array_equal(y0, g["y0"]) and np.array_equal(y1, g["y1"])
    mo = (1 << g["bo"]) - 1
    gs = g["g"]
    hit = np.repeat(g["maskedX"].astype(object) == g["alpha"].astype(object), gs)
    y = (y0.astype(object) + y1.astype(object)) & mo
    assert all(int(a) == ((int(b) & mo) if h else 0) for a, b, h in zip(y, g["beta"], hit))


def test_dpf_eval_all_golden(oracle):
    g = load_golden("dpf_eval_all_u8_n6_g2")
    for p in (0, 1):
        y = oracle.dpf_eval_all(g["maskedX"], g["key"], g[f"seed{p}"], p, g["n"], g["bo"], g["g"])
        assert np.array_equal(y, g[f"y{p}"])


def test_dpf_eval_multi_golden(oracle):
    g = load_golden("dpf_eval_multi_u16_n10")
    for p in (0, 1):
        y = oracle.dpf_eval_multi(g["maskedX"], g["key"], g[f"seed{p}"], p, g["point"], g["n"], g["bo"], g["g"])
        assert np.array_equal(y, g[f"y{p}"])


@pytest.mark.parametrize("name", golden_names("grotto_u"))
def test_grotto_golden(oracle, name):
    g = load_golden(name)
    n = g["n"]
    key = oracle.grotto_keygen(g["alpha"], g["seed0"], g["seed1"], n)
    assert np.array_equal(key, g["key"])
    for p in (0, 1):
        s = g[f"seed{p}"]
        assert np.array_equal(oracle.grotto_eq_eval(g["maskedX"], key, s, p, n), g[f"eq{p}"])
        assert np.array_equal(oracle.grotto_eval(g["maskedX"], key, s, False, p, n), g[f"lt{p}"])
        assert np.array_equal(oracle.grotto_eval(g["maskedX"], key, s, True, p, n), g[f"le{p}"])
        assert np.array_equal(oracle.grotto_mic_eval(g["maskedX"], key, s, p, g["left"], g["right"], n), g[f"mic{p}"])
        e, t = oracle.grotto_interval_lut_eval(g["maskedX"], key, s, p, g["left"], g["right"], g["lut"], n,
                                               8 * g["es"])
        assert np.array_equal(e, g[f"lutE{p}"]) and np.array_equal(t, g[f"lutT{p}"])
    # reconstruction (tests/grotto/grotto_eval_test_case.h:60-66)
    x = g["maskedX"].astype(object) % (1 << n)
    a = g["alpha"].astype(object)
    assert all(int(u) == int(v) for u, v in zip((g["eq0"] ^ g["eq1"]) & 1, x == a))
    assert all(int(u) == int(v) for u, v in zip((g["lt0"] ^ g["lt1"]) & 1, x < a))
    assert all(int(u) == int(v) for u, v in zip((g["le0"] ^ g["le1"]) & 1, x <= a))


def test_grotto_full_domain_golden(oracle):
    g = load_golden("grotto_all_u16_n10")
    N = g["alpha"].size
    for p in (0, 1):
        assert np.array_equal(oracle.grotto_eq_eval_all(g["key"], g[f"seed{p}"], p, g["n"], g["es"], N), g[f"eqbits{p}"])
        assert np.array_equal(oracle.grotto_le_eval_all(g["key"], g[f"seed{p}"], p, g["n"], g["es"], N), g[f"lebits{p}"])
    dom = 1 << g["n"]
    eq = np.unpackbits(g["eqbits0"] ^ g["eqbits1"], bitorder="little").reshape(N, dom)
    assert np.array_equal(eq.argmax(axis=1), g["alpha"].astype(np.int64)) and eq.sum() == N


@pytest.mark.parametrize("name", golden_names("dcf_mic_u"))
def test_dcf_mic_golden(oracle, name):
    g = load_golden(name)
    key, z = oracle.dcf_mic_keygen(g["alpha"], g["seed0"], g["seed1"], g["left"], g["right"], g["n"], g["bo"])
    assert np.array_equal(key, g["key"]) and np.array_equal(z, g["z"])
    for p in (0, 1):
        y = oracle.dcf_mic_eval(g["maskedX"], key, g[f"z{p}"], g[f"seed{p}"], p, g["left"], g["right"], g["n"], g["bo"])
        assert np.array_equal(y, g[f"y{p}"])


@pytest.mark.parametrize("name", golden_names("spline_u"))
def test_spline_golden(oracle, name):
    g = load_golden(name)
    key, e, beta = oracle.spline_keygen(g["alpha"], g["seed0"], g["seed1"], g["coeffs"], g["d"], g["left"], g["right"],
                                        g["n"], g["bo"])
    assert np.array_equal(key, g["key"]) and np.array_equal(e, g["e"]) and np.array_equal(beta, g["beta"])
    for p in (0, 1):
        y = oracle.spline_eval(g["maskedX"], key, g[f"e{p}"], g[f"b{p}"], g[f"seed{p}"], p, g["left"], g["right"],
                               g["d"], g["n"], g["bo"])
        assert np.array_equal(y, g[f"y{p}"])


@pytest.mark.parametrize("name", golden_names("ottt_u"))
def test_ottt_golden(oracle, name):
    g = load_golden(name)
    assert np.array_equal(oracle.ottt_keygen(g["key0"], g["alpha"], g["n"]), g["key1"])
    for p in (0, 1):
        e, t = oracle.ottt_lut_eval(g["maskedX"], g[f"key{p}"], p, g["lut"], g["n"])
        assert np.array_equal(e, g[f"e{p}"]) and np.array_equal(t, g[f"t{p}"])


# ---------------- fresh random cases against the reference library itself ----------------

WIDTHS = [(es, n, bo) for es in (1, 2, 4, 8) for n in sorted({1, 8 * es - 1, 8 * es})
          for bo in sorted({1, 8 * es - 1, 8 * es})]


@pytest.mark.parametrize("es,n,bo", WIDTHS)
@pytest.mark.parametrize("g", [1, 2, 3])
def test_dcf_dpf_vs_reference(oracle, refcpu, es, n, bo, g):
    rng = np.random.default_rng(es * 1000 + n * 10 + bo + g * 7)
    N = 33
    a, b, s0, s1 = rnd(rng, N, es, n), rnd(rng, N * g, es, bo), seeds(rng, N), seeds(rng, N)
    x = rnd(rng, N, es, 8 * es)
    for kg, ev in (("dcf_keygen", "dcf_eval"), ("dpf_keygen", "dpf_eval")):
        k = getattr(oracle, kg)(a, b, s0, s1, n, bo, g)
        assert np.array_equal(k, getattr(refcpu, kg)(a, b, s0, s1, n, bo, g))
        for p, s in ((0, s0), (1, s1)):
            assert np.array_equal(getattr(oracle, ev)(x, k, s, p, n, bo, g), getattr(refcpu, ev)(x, k, s, p, n, bo, g))


@pytest.mark.parametrize("es", [1, 2, 4, 8])
def test_grotto_mic_spline_vs_reference(oracle, refcpu, es):
    rng = np.random.default_rng(77 + es)
    W = 8 * es
    for n in sorted({6, W - 1, W} if W >= 8 else {6, 7, 8}):
        if n < 6 or n > W:
            continue
        N = 21
        a, s0, s1 = rnd(rng, N, es, n), seeds(rng, N), seeds(rng, N)
        k = oracle.grotto_keygen(a, s0, s1, n)
        assert np.array_equal(k, refcpu.grotto_keygen(a, s0, s1, n))
        x = rnd(rng, N, es, W)
        L, R = random_intervals(rng, 4, es, n)
        for p, s in ((0, s0), (1, s1)):
            for eb in (False, True):
                assert np.array_equal(oracle.grotto_eval(x, k, s, eb, p, n), refcpu.grotto_eval(x, k, s, eb, p, n))
            assert np.array_equal(oracle.grotto_mic_eval(x, k, s, p, L, R, n), refcpu.grotto_mic_eval(x, k, s, p, L, R, n))
    n = bo = W
    N, m, d = 5, 3, 2
    a, s0, s1 = rnd(rng, N, es, n), seeds(rng, N), seeds(rng, N)
    L, R = sorted_partition(rng, m, es, n)
    c = rnd(rng, m * (d + 1), es, W)
    ko = oracle.spline_keygen(a, s0, s1, c, d, L, R, n, bo)
    kr = refcpu.spline_keygen(a, s0, s1, c, d, L, R, n, bo)
    assert all(np.array_equal(u, v) for u, v in zip(ko, kr))
    x = rnd(rng, N, es, W)
    for p, s in ((0, s0), (1, s1)):
        assert np.array_equal(oracle.spline_eval(x, ko[0], ko[1], ko[2], s, p, L, R, d, n, bo),
                              refcpu.spline_eval(x, ko[0], ko[1], ko[2], s, p, L, R, d, n, bo))
