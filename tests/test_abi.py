"""The drop-in boundary, without a GPU: the library loads, exports every symbol the headers
declare, answers the host-side size queries like the reference library, and validates
arguments with the reference's error codes in the reference's order (every case here is
invalid, so no call reaches device work)."""

import ctypes
import glob
import itertools
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    from fastfunctionsecretsharing_b200 import _lib

    if not os.path.exists(_lib.LIB_PATH):
        from fastfunctionsecretsharing_b200.build import build

        build()
    return _lib.load()


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "FastFss", "**", "*.h"), recursive=True):
        txt = open(h).read()
        names.update(re.findall(r"FAST_FSS_API\s+[\w\s\*]+?\b(FastFss_\w+)\s*\(", txt))
    return sorted(names)


def test_exports_every_declared_symbol(lib):
    names = declared_symbols()
    assert len(names) >= 52  # 52 reference symbols + this library's extensions
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_reference_symbols_are_declared():
    """Every FastFss_cuda_* / host symbol of the reference ABI is declared here too."""
    ours = set(declared_symbols())
    reference_abi = {
        "FastFss_cuda_dcfKeyGen", "FastFss_cuda_dcfEval", "FastFss_cuda_dpfKeyGen", "FastFss_cuda_dpfEval",
        "FastFss_cuda_dpfEvalAll", "FastFss_cuda_dpfEvalMulti", "FastFss_cuda_grottoKeyGen",
        "FastFss_cuda_grottoEqEval", "FastFss_cuda_grottoEval", "FastFss_cuda_grottoMICEval",
        "FastFss_cuda_grottoIntervalLutEval", "FastFss_cuda_dcfMICKeyGen", "FastFss_cuda_dcfMICEval",
        "FastFss_cuda_dcfSplineKeyGen", "FastFss_cuda_dcfSplineEval", "FastFss_cuda_otttKeyGen",
        "FastFss_cuda_otttLutEval", "FastFss_cuda_setGridDim", "FastFss_cuda_getGridDim",
        "FastFss_cuda_getFineGrainParallelGridDimThreshold", "FastFss_cuda_setFineGrainParallelGridDimThreshold",
        "FastFss_cuda_prngInit", "FastFss_cuda_prngRelease", "FastFss_cuda_prngSetCurrentSeed",
        "FastFss_cuda_prngGetCurrentSeed", "FastFss_cuda_prngGen", "FastFss_otttGetKeyDataSize",
    }
    for algo in ("dcf", "dpf", "grotto", "dcfMIC", "dcfSpline"):
        reference_abi |= {f"FastFss_{algo}KeyZip", f"FastFss_{algo}KeyUnzip", f"FastFss_{algo}GetKeyDataSize",
                          f"FastFss_{algo}GetZippedKeyDataSize", f"FastFss_{algo}GetCacheDataSize"}
    assert reference_abi <= ours, sorted(reference_abi - ours)


def test_config_knobs(lib):
    assert lib.FastFss_cuda_getGridDim() == 128
    assert lib.FastFss_cuda_getFineGrainParallelGridDimThreshold() == 64
    assert lib.FastFss_cuda_setGridDim(0) == -2 and lib.FastFss_cuda_setGridDim(-5) == -2
    assert lib.FastFss_cuda_setGridDim(256) == 0 and lib.FastFss_cuda_getGridDim() == 256
    assert lib.FastFss_cuda_setGridDim(128) == 0
    assert lib.FastFss_cuda_setFineGrainParallelGridDimThreshold(0) == -2
    assert lib.FastFss_cuda_setFineGrainParallelGridDimThreshold(64) == 0


def test_zip_stubs(lib):
    assert lib.FastFss_dcfKeyZip(None, 0, None, 0, 8, 8, 1, 1, 1) == -1
    assert lib.FastFss_dpfKeyUnzip(None, 0, None, 0, 8, 8, 1, 1, 1) == -1
    assert lib.FastFss_grottoKeyZip(None, 0, None, 0, 8, 1, 1) == -1


SIZE_QUERIES = {
    # name: argument tuples after the out pointer
    "FastFss_dcfGetKeyDataSize": [(n, bo, g, es, N) for n in (0, 1, 8, 9, 32, 64, 65) for bo in (0, 8, 33)
                                  for g in (0, 1, 3) for es in (1, 2, 3, 4, 8) for N in (0, 5)],
    "FastFss_dcfGetZippedKeyDataSize": [(n, 8, 1, es, 3) for n in (0, 8, 9) for es in (1, 3, 8)],
    "FastFss_dcfGetCacheDataSize": [(n, bo, g, es, 7) for n in (0, 5, 8, 9) for bo in (0, 8) for g in (1, 4)
                                    for es in (1, 2, 5, 8)],
    "FastFss_dpfGetKeyDataSize": [(n, bo, g, es, N) for n in (0, 1, 16, 17) for bo in (0, 16, 17) for g in (0, 2)
                                  for es in (2, 3, 4) for N in (0, 9)],
    "FastFss_dpfGetZippedKeyDataSize": [(n, 8, 1, es, 3) for n in (0, 8, 9) for es in (1, 7)],
    "FastFss_grottoGetKeyDataSize": [(n, es, N) for n in (5, 6, 7, 16, 17, 64) for es in (1, 2, 8, 6) for N in (0, 4)],
    "FastFss_grottoGetZippedKeyDataSize": [(n, es, 4) for n in (5, 6, 16) for es in (1, 2, 6)],
    "FastFss_grottoGetCacheDataSize": [(n, es, 4) for n in (5, 6, 16) for es in (2, 6, 8)],
    "FastFss_dcfMICGetKeyDataSize": [(n, bo, es, 3) for n in (1, 16) for bo in (4, 16) for es in (2, 3, 8)],
    "FastFss_dcfMICGetCacheDataSize": [(n, bo, es, 3) for n in (1, 16) for bo in (4, 16) for es in (2, 3)],
    "FastFss_dcfMICGetZippedKeyDataSize": [(16, 16, es, 3) for es in (2, 3)],
    "FastFss_dcfSplineGetKeyDataSize": [(d, m, n, bo, es, N) for d in (0, 2) for m in (1, 32) for n in (16, 64)
                                        for bo in (64,) for es in (8, 3, 4) for N in (1, 10)],
    "FastFss_dcfSplineGetCacheDataSize": [(d, m, n, 64, es, 10) for d in (0, 2) for m in (1, 32) for n in (16, 64)
                                          for es in (8, 3)],
    "FastFss_dcfSplineGetZippedKeyDataSize": [(2, 4, 64, 64, es, 2) for es in (8, 3)],
    "FastFss_otttGetKeyDataSize": [(n, N) for n in (2, 3, 8, 20) for N in (0, 3)],
}


# The reference CPU library here is built without the wide-integer widths (its wideint
# dependency is absent), so 16/24/32-byte elements are checked against the size formulas.
def test_size_queries_wide_elements(lib):
    for es in (16, 24, 32):
        v = ctypes.c_size_t(0)
        assert lib.FastFss_dcfGetKeyDataSize(ctypes.byref(v), 100, 70, 3, es, 7) == 0
        assert v.value == 7 * (16 * 100 + es * 100 * 3 + 2 * es + es * 3)
        assert lib.FastFss_dcfGetCacheDataSize(ctypes.byref(v), 100, 70, 3, es, 7) == 0
        assert v.value == 7 * 16 * 100 + 7 * es * 100 * 3
        assert lib.FastFss_dpfGetCacheDataSize(ctypes.byref(v), 100, es, 7) == 0 and v.value == 7 * 1600
        assert lib.FastFss_grottoGetKeyDataSize(ctypes.byref(v), 100, es, 7) == 0
        assert v.value == 7 * (16 * 94 + 8 + 2 * es)


@pytest.mark.parametrize("name", sorted(SIZE_QUERIES))
def test_size_queries_match_reference(lib, refcpu, name):
    mine, ref = getattr(lib, name), getattr(refcpu.lib, name)
    for args in SIZE_QUERIES[name]:
        a, b = ctypes.c_size_t(12345), ctypes.c_size_t(12345)
        ca = [ctypes.c_size_t(v) for v in args]
        ra = mine(ctypes.byref(a), *ca)
        rb = ref(ctypes.byref(b), *ca)
        assert ra == rb, (name, args)
        assert a.value == b.value, (name, args, a.value, b.value)


# ----------------------------------------------------------------------------------------
# Validation order: every corrupted call must fail with the reference's code.
# ----------------------------------------------------------------------------------------

BUF = ctypes.create_string_buffer(64)
P = ctypes.cast(BUF, ctypes.c_void_p)


def sz(v):
    return ctypes.c_size_t(v)


def call(fn, spec, vals, cuda):
    args = []
    for kind, name in spec:
        v = vals[name]
        if kind == "p":
            args.append(P if v else None)
        elif kind == "i":
            args.append(ctypes.c_int(v))
        elif kind == "b":
            args.append(ctypes.c_bool(v))
        else:
            args.append(sz(v))
    if cuda:
        args.append(None)
    return fn(*args)


def dcf_key(n, g, es, N):
    return N * (16 * n + es * n * g + 2 * es + es * g)


def dpf_key(n, g, es, N):
    return N * (16 * n + 2 * es + es * g)


def grotto_key(n, es, N):
    return N * (16 * (n - 6) + 8 + 2 * es)


CASES = {}

es, n, bo, g, N = 4, 20, 24, 2, 5
CASES["dcfKeyGen"] = (
    [("p", "key"), ("s", "keyN"), ("p", "alpha"), ("s", "alphaN"), ("p", "beta"), ("s", "betaN"), ("p", "s0"),
     ("s", "s0N"), ("p", "s1"), ("s", "s1N"), ("s", "n"), ("s", "bo"), ("s", "g"), ("s", "es"), ("s", "N")],
    dict(key=1, keyN=dcf_key(n, g, es, N), alpha=1, alphaN=N * es, beta=1, betaN=N * es * g, s0=1, s0N=16 * N, s1=1,
         s1N=16 * N, n=n, bo=bo, g=g, es=es, N=N),
    dict(keyN=1, alphaN=1, betaN=3, s0N=1, s1N=1, n=[0, 33], bo=[0, 40], g=0))
CASES["dcfEval"] = (
    [("p", "out"), ("s", "outN"), ("p", "x"), ("s", "xN"), ("p", "key"), ("s", "keyN"), ("p", "seed"), ("s", "seedN"),
     ("i", "party"), ("s", "n"), ("s", "bo"), ("s", "g"), ("s", "es"), ("s", "N"), ("p", "cache"), ("s", "cacheN")],
    dict(out=1, outN=N * es * g, x=1, xN=N * es, key=1, keyN=dcf_key(n, g, es, N), seed=1, seedN=16 * N, party=1, n=n,
         bo=bo, g=g, es=es, N=N, cache=0, cacheN=0),
    dict(outN=1, xN=1, keyN=1, seedN=1, party=[2, -1], n=[0, 33], bo=[0, 33], g=0, cacheN=5))
CASES["dpfKeyGen"] = (
    CASES["dcfKeyGen"][0],
    dict(key=1, keyN=dpf_key(n, g, es, N), alpha=1, alphaN=N * es, beta=1, betaN=N * es * g, s0=1, s0N=16 * N, s1=1,
         s1N=16 * N, n=n, bo=bo, g=g, es=es, N=N),
    dict(keyN=1, alphaN=1, betaN=[3, 0], s0N=1, s1N=1, n=[0, 33], bo=[0, 40], g=0))
CASES["dpfEval"] = (
    CASES["dcfEval"][0],
    dict(out=1, outN=N * es * g, x=1, xN=N * es, key=1, keyN=dpf_key(n, g, es, N), seed=1, seedN=16 * N, party=0,
         n=n, bo=bo, g=g, es=es, N=N, cache=0, cacheN=0),
    dict(outN=1, xN=1, keyN=1, seedN=1, party=2, n=[0, 33], bo=[0, 33], g=0, cacheN=5))
CASES["dpfEvalAll"] = (
    CASES["dcfEval"][0],
    dict(out=1, outN=N * es * (1 << 6) * g, x=1, xN=N * es, key=1, keyN=dpf_key(6, g, es, N), seed=1, seedN=16 * N,
         party=0, n=6, bo=bo, g=g, es=es, N=N, cache=0, cacheN=0),
    dict(outN=1, xN=1, keyN=1, seedN=1, party=2, n=[0, 33], bo=[0, 33], g=0, cacheN=5))
CASES["dpfEvalMulti"] = (
    [("p", "out"), ("s", "outN"), ("p", "x"), ("s", "xN"), ("p", "key"), ("s", "keyN"), ("p", "seed"), ("s", "seedN"),
     ("i", "party"), ("p", "pt"), ("s", "ptN"), ("s", "n"), ("s", "bo"), ("s", "g"), ("s", "es"), ("s", "N"),
     ("p", "cache"), ("s", "cacheN")],
    dict(out=1, outN=N * es * 3 * g, x=1, xN=N * es, key=1, keyN=dpf_key(n, g, es, N), seed=1, seedN=16 * N,
         party=1, pt=1, ptN=3 * es, n=n, bo=bo, g=g, es=es, N=N, cache=0, cacheN=0),
    dict(outN=1, xN=1, keyN=1, seedN=1, party=2, ptN=[5, 8], n=[0, 33], bo=0, g=0, cacheN=5))
ng = 16
CASES["grottoKeyGen"] = (
    [("p", "key"), ("s", "keyN"), ("p", "alpha"), ("s", "alphaN"), ("p", "s0"), ("s", "s0N"), ("p", "s1"),
     ("s", "s1N"), ("s", "n"), ("s", "es"), ("s", "N")],
    dict(key=1, keyN=grotto_key(ng, es, N), alpha=1, alphaN=N * es, s0=1, s0N=16 * N, s1=1, s1N=16 * N, n=ng, es=es,
         N=N),
    dict(keyN=1, alphaN=1, s0N=1, s1N=1, n=[5, 33]))
CASES["grottoEqEval"] = (
    [("p", "out"), ("s", "outN"), ("p", "x"), ("s", "xN"), ("p", "key"), ("s", "keyN"), ("p", "seed"), ("s", "seedN"),
     ("i", "party"), ("s", "n"), ("s", "es"), ("s", "N"), ("p", "cache"), ("s", "cacheN")],
    dict(out=1, outN=N * es, x=1, xN=N * es, key=1, keyN=grotto_key(ng, es, N), seed=1, seedN=16 * N, party=0, n=ng,
         es=es, N=N, cache=0, cacheN=0),
    dict(outN=1, xN=1, keyN=1, seedN=1, party=2, n=[5, 33], cacheN=5))
CASES["grottoEval"] = (
    [("p", "out"), ("s", "outN"), ("p", "x"), ("s", "xN"), ("p", "key"), ("s", "keyN"), ("p", "seed"), ("s", "seedN"),
     ("b", "eb"), ("i", "party"), ("s", "n"), ("s", "es"), ("s", "N"), ("p", "cache"), ("s", "cacheN")],
    dict(CASES["grottoEqEval"][1], eb=True),
    dict(outN=1, xN=1, keyN=1, seedN=1, party=2, n=[5, 33], cacheN=5))
CASES["grottoMICEval"] = (
    [("p", "out"), ("s", "outN"), ("p", "x"), ("s", "xN"), ("p", "key"), ("s", "keyN"), ("p", "seed"), ("s", "seedN"),
     ("i", "party"), ("p", "L"), ("s", "LN"), ("p", "R"), ("s", "RN"), ("s", "n"), ("s", "es"), ("s", "N"),
     ("p", "cache"), ("s", "cacheN")],
    dict(out=1, outN=N * es * 3, x=1, xN=N * es, key=1, keyN=grotto_key(ng, es, N), seed=1, seedN=16 * N, party=1,
         L=1, LN=3 * es, R=1, RN=3 * es, n=ng, es=es, N=N, cache=0, cacheN=0),
    dict(outN=1, xN=1, keyN=1, seedN=1, party=2, LN=[5, 8], RN=[5, 8], n=[5, 33], cacheN=5))
CASES["grottoIntervalLutEval"] = (
    [("p", "oe"), ("s", "oeN"), ("p", "ot"), ("s", "otN"), ("p", "x"), ("s", "xN"), ("p", "key"), ("s", "keyN"),
     ("p", "seed"), ("s", "seedN"), ("i", "party"), ("p", "L"), ("s", "LN"), ("p", "R"), ("s", "RN"), ("p", "lut"),
     ("s", "lutN"), ("s", "n"), ("s", "bo"), ("s", "es"), ("s", "N"), ("p", "cache"), ("s", "cacheN")],
    dict(oe=1, oeN=N * es, ot=1, otN=N * es * 2, x=1, xN=N * es, key=1, keyN=grotto_key(ng, es, N), seed=1,
         seedN=16 * N, party=0, L=1, LN=3 * es, R=1, RN=3 * es, lut=1, lutN=3 * es * 2, n=ng, bo=16, es=es, N=N,
         cache=0, cacheN=0),
    dict(oeN=1, otN=1, xN=1, keyN=1, seedN=1, party=2, LN=[5, 8], RN=8, lutN=[5, 3 * es * 3], n=[5, 33], cacheN=5))
CASES["dcfMICKeyGen"] = (
    [("p", "key"), ("s", "keyN"), ("p", "z"), ("s", "zN"), ("p", "alpha"), ("s", "alphaN"), ("p", "s0"), ("s", "s0N"),
     ("p", "s1"), ("s", "s1N"), ("p", "L"), ("s", "LN"), ("p", "R"), ("s", "RN"), ("s", "n"), ("s", "bo"), ("s", "es"),
     ("s", "N")],
    dict(key=1, keyN=dcf_key(n, 1, es, N), z=1, zN=N * es * 3, alpha=1, alphaN=N * es, s0=1, s0N=16 * N, s1=1,
         s1N=16 * N, L=1, LN=3 * es, R=1, RN=3 * es, n=n, bo=bo, es=es, N=N),
    dict(keyN=1, zN=1, alphaN=1, s0N=1, s1N=1, LN=[5, 8], RN=5, n=[0, 33], bo=[0, 33]))
CASES["dcfMICEval"] = (
    [("p", "out"), ("s", "outN"), ("p", "x"), ("s", "xN"), ("p", "key"), ("s", "keyN"), ("p", "z"), ("s", "zN"),
     ("p", "seed"), ("s", "seedN"), ("i", "party"), ("p", "L"), ("s", "LN"), ("p", "R"), ("s", "RN"), ("s", "n"),
     ("s", "bo"), ("s", "es"), ("s", "N"), ("p", "cache"), ("s", "cacheN")],
    dict(out=1, outN=N * es * 3, x=1, xN=N * es, key=1, keyN=dcf_key(n, 1, es, N), z=1, zN=N * es * 3, seed=1,
         seedN=16 * N, party=1, L=1, LN=3 * es, R=1, RN=3 * es, n=n, bo=bo, es=es, N=N, cache=0, cacheN=0),
    dict(outN=1, xN=1, keyN=1, zN=1, seedN=1, party=2, LN=[5, 8], RN=5, n=[0, 33], bo=0, cacheN=5))
m, d = 3, 2
gs = m * (d + 1)
CASES["dcfSplineKeyGen"] = (
    [("p", "key"), ("s", "keyN"), ("p", "e"), ("s", "eN"), ("p", "beta"), ("s", "betaN"), ("p", "alpha"),
     ("s", "alphaN"), ("p", "s0"), ("s", "s0N"), ("p", "s1"), ("s", "s1N"), ("p", "c"), ("s", "cN"), ("s", "d"),
     ("p", "L"), ("s", "LN"), ("p", "R"), ("s", "RN"), ("s", "m"), ("s", "n"), ("s", "bo"), ("s", "es"), ("s", "N")],
    dict(key=1, keyN=dcf_key(n, gs, es, N), e=1, eN=N * es * gs, beta=1, betaN=N * es * gs, alpha=1, alphaN=N * es,
         s0=1, s0N=16 * N, s1=1, s1N=16 * N, c=1, cN=gs * es, d=d, L=1, LN=m * es, R=1, RN=m * es, m=m, n=n, bo=bo,
         es=es, N=N),
    dict(keyN=1, eN=1, betaN=1, alphaN=1, s0N=1, s1N=1, cN=1, LN=1, RN=1, m=0, n=[0, 33], bo=[0, 33]))
CASES["dcfSplineEval"] = (
    [("p", "out"), ("s", "outN"), ("p", "x"), ("s", "xN"), ("p", "key"), ("s", "keyN"), ("p", "e"), ("s", "eN"),
     ("p", "beta"), ("s", "betaN"), ("p", "seed"), ("s", "seedN"), ("i", "party"), ("p", "L"), ("s", "LN"),
     ("p", "R"), ("s", "RN"), ("s", "m"), ("s", "d"), ("s", "n"), ("s", "bo"), ("s", "es"), ("s", "N"),
     ("p", "cache"), ("s", "cacheN")],
    dict(out=1, outN=N * es, x=1, xN=N * es, key=1, keyN=dcf_key(n, gs, es, N), e=1, eN=N * es * gs, beta=1,
         betaN=N * es * gs, seed=1, seedN=16 * N, party=0, L=1, LN=m * es, R=1, RN=m * es, m=m, d=d, n=n, bo=bo,
         es=es, N=N, cache=1,
         cacheN=N * 16 * n + N * es * n * gs + N * es * (2 * gs + d + 1)),
    dict(outN=1, xN=1, keyN=1, eN=1, betaN=1, seedN=1, party=2, LN=1, RN=1, m=0, n=[0, 33], bo=[0, 33], cache=0,
         cacheN=[0, 7]))
CASES["otttKeyGen"] = (
    [("p", "key"), ("s", "keyN"), ("p", "alpha"), ("s", "alphaN"), ("s", "n"), ("s", "es"), ("s", "N")],
    dict(key=1, keyN=N * (1 << 10) // 8, alpha=1, alphaN=N * es, n=10, es=es, N=N),
    dict(keyN=1, alphaN=1, n=[2, 33]))
CASES["otttLutEval"] = (
    [("p", "oe"), ("s", "oeN"), ("p", "ot"), ("s", "otN"), ("p", "x"), ("s", "xN"), ("p", "key"), ("s", "keyN"),
     ("i", "party"), ("p", "lut"), ("s", "lutN"), ("s", "n"), ("s", "es"), ("s", "N")],
    dict(oe=1, oeN=N * es, ot=1, otN=N * es * 2, x=1, xN=N * es, key=1, keyN=N * (1 << 10) // 8, party=0, lut=1,
         lutN=2 * es * (1 << 10), n=10, es=es, N=N),
    dict(oeN=1, otN=1, xN=1, keyN=1, party=2, lutN=[5, 3 * es * (1 << 10)], n=[2, 33]))


def corruptions(bad):
    single = []
    for k, v in bad.items():
        for val in (v if isinstance(v, list) else [v]):
            single.append((k, val))
    return single


@pytest.mark.parametrize("api", sorted(CASES))
def test_validation_order_matches_reference(lib, refcpu, api):
    spec, base, bad = CASES[api]
    mine = getattr(lib, f"FastFss_cuda_{api}")
    ref = getattr(refcpu.lib, f"FastFss_cpu_{api}")
    single = corruptions(bad)
    checked = 0
    for combo in itertools.chain(((c,) for c in single), itertools.combinations(single, 2)):
        if len({k for k, _ in combo}) < len(combo):
            continue
        vals = dict(base)
        for k, v in combo:
            vals[k] = v
        rb = call(ref, spec, vals, cuda=False)
        assert rb != 0, (api, combo)  # every case is invalid for the reference
        ra = call(mine, spec, vals, cuda=True)
        assert ra == rb, (api, combo, ra, rb)
        checked += 1
    assert checked > len(single)


def test_unsupported_element_size(lib):
    for es in (3, 16):
        rc = lib.FastFss_cuda_dcfEval(None, 0, None, 0, None, 0, None, 0, 0, 8, 8, 1, es, 1, None, 0, None)
        assert rc == -11


def test_misaligned_key_or_seed_is_refused(lib):
    """Keys and seeds are read as 16-byte vectors: a key or seed pointer that is 8 but not 16
    byte aligned is refused (FAST_FSS_RUNTIME_ERROR) after the reference's own checks pass and
    before anything is launched (the pointers here are host addresses and are never read)."""
    base = ctypes.addressof(BUF)
    off = (8 - base) % 16  # base + off is 8 mod 16: aligned for every ring element, not for blocks
    mis = ctypes.c_void_p(base + off)
    for api, (spec, vals, _bad) in sorted(CASES.items()):
        if api.startswith("ottt"):
            continue  # OTTT keys are bit rows, read at byte/word granularity
        args = []
        for kind, name in spec:
            v = vals[name]
            if kind == "p":
                args.append(mis)
            elif kind == "i":
                args.append(ctypes.c_int(v))
            elif kind == "b":
                args.append(ctypes.c_bool(v))
            else:
                args.append(sz(v))
        args.append(None)
        assert getattr(lib, f"FastFss_cuda_{api}")(*args) == -1, api
