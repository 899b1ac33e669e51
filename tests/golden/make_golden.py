"""Regenerates the golden fixtures in this directory from the reference's own CPU code.

    make -C oracle ref           # builds oracle/_ref/libfastfss_ref.so from the reference sources
    python tests/golden/make_golden.py

Every fixture holds seeded inputs and the outputs of the reference library's FastFss_cpu_*
entry points (src/cpu/*.cpp compiled where they lie) for them: keys byte for byte and both
parties' shares. The fixtures pin the oracle restatement (tests/test_oracle_pin.py) and the
CUDA library (tests/test_gpu_*.py) without the reference tree being present.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle.pyoracle import RefCpu  # noqa: E402
from fss_cases import (DTYPES, dcf_regions, grotto_regions, random_intervals, rnd, seeds,  # noqa: E402
                       sorted_partition, take_elements)


def save(name, **arrays):
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
    print(name, sum(a.nbytes for a in arrays.values() if isinstance(a, np.ndarray)), "bytes")


def dcf_case(R, rng, name, es, n, bo, g, N):
    a, b = rnd(rng, N, es, n), rnd(rng, N * g, es, bo)
    s0, s1 = seeds(rng, N), seeds(rng, N)
    key = R.dcf_keygen(a, b, s0, s1, n, bo, g)
    x = rnd(rng, N, es, n)
    mx = ((x.astype(np.uint64) + a.astype(np.uint64)) & np.uint64((1 << n) - 1 if n < 64 else 2**64 - 1)).astype(
        DTYPES[es])
    y0 = R.dcf_eval(mx, key, s0, 0, n, bo, g)
    y1 = R.dcf_eval(mx, key, s1, 1, n, bo, g)
    save(name, es=es, n=n, bo=bo, g=g, alpha=a, beta=b, seed0=s0, seed1=s1, key=key, maskedX=mx, y0=y0, y1=y1)


def dpf_case(R, rng, name, es, n, bo, g, N):
    a, b = rnd(rng, N, es, n), rnd(rng, N * g, es, bo)
    s0, s1 = seeds(rng, N), seeds(rng, N)
    key = R.dpf_keygen(a, b, s0, s1, n, bo, g)
    x = rnd(rng, N, es, n)
    x[::3] = 0  # every third element hits alpha (tests/dpf/dpf_eval_case.h:72-74)
    mx = ((x.astype(np.uint64) + a.astype(np.uint64)) & np.uint64((1 << n) - 1 if n < 64 else 2**64 - 1)).astype(
        DTYPES[es])
    y0 = R.dpf_eval(mx, key, s0, 0, n, bo, g)
    y1 = R.dpf_eval(mx, key, s1, 1, n, bo, g)
    save(name, es=es, n=n, bo=bo, g=g, alpha=a, beta=b, seed0=s0, seed1=s1, key=key, maskedX=mx, y0=y0, y1=y1)


def main():
    R = RefCpu()
    rng = np.random.default_rng(20261203)

    # DCF: BASELINE config-1 shape (n=16 over u16), config-2 shape (n=32 over u32) and the
    # width / group-size corners of tests/dcf/dcf_eval_cuda.cu:250-306.
    dcf_case(R, rng, "dcf_u16_n16_g1", 2, 16, 16, 1, 128)
    dcf_case(R, rng, "dcf_u32_n32_g1", 4, 32, 32, 1, 64)
    dcf_case(R, rng, "dcf_u8_n7_g3", 1, 7, 8, 3, 64)
    dcf_case(R, rng, "dcf_u64_n64_bo63_g2", 8, 64, 63, 2, 24)
    dcf_case(R, rng, "dcf_u64_n63_g3_aes", 8, 63, 64, 3, 16)
    dcf_case(R, rng, "dcf_u32_n1_bo1_g4", 4, 1, 1, 4, 64)

    # DPF, incl. the leaf-convert argument order (ceil(g/8) bytes per value).
    dpf_case(R, rng, "dpf_u32_n32_g1", 4, 32, 32, 1, 64)
    dpf_case(R, rng, "dpf_u16_n12_g3", 2, 12, 16, 3, 64)
    dpf_case(R, rng, "dpf_u64_n64_g2", 8, 64, 64, 2, 24)
    dpf_case(R, rng, "dpf_u8_n8_bo1_g1", 1, 8, 1, 1, 64)

    # DPF full domain and multi-point.
    es, n, bo, g, N = 1, 6, 8, 2, 8
    a, b = rnd(rng, N, es, n), rnd(rng, N * g, es, bo)
    s0, s1 = seeds(rng, N), seeds(rng, N)
    key = R.dpf_keygen(a, b, s0, s1, n, bo, g)
    mx = rnd(rng, N, es, 8)
    save("dpf_eval_all_u8_n6_g2", es=es, n=n, bo=bo, g=g, alpha=a, beta=b, seed0=s0, seed1=s1, key=key, maskedX=mx,
         y0=R.dpf_eval_all(mx, key, s0, 0, n, bo, g), y1=R.dpf_eval_all(mx, key, s1, 1, n, bo, g))
    es, n, bo, g, N = 2, 10, 16, 1, 16
    a, b = rnd(rng, N, es, n), rnd(rng, N * g, es, bo)
    s0, s1 = seeds(rng, N), seeds(rng, N)
    key = R.dpf_keygen(a, b, s0, s1, n, bo, g)
    mx = rnd(rng, N, es, 16)
    pt = rnd(rng, 5, es, 16)
    pt[0] = np.uint16((int(mx[0]) - int(a[0])) % 65536)
    save("dpf_eval_multi_u16_n10", es=es, n=n, bo=bo, g=g, alpha=a, beta=b, seed0=s0, seed1=s1, key=key,
         maskedX=mx, point=pt, y0=R.dpf_eval_multi(mx, key, s0, 0, pt, n, bo, g),
         y1=R.dpf_eval_multi(mx, key, s1, 1, pt, n, bo, g))

    # Grotto: keys, eq / lt / le shares, MIC and interval LUT (BASELINE config-3 shape n=16).
    for es, n, N, m in ((2, 16, 64, 8), (8, 64, 24, 5), (1, 7, 32, 3)):
        a = rnd(rng, N, es, n)
        s0, s1 = seeds(rng, N), seeds(rng, N)
        key = R.grotto_keygen(a, s0, s1, n)
        mx = rnd(rng, N, es, 8 * es)
        mx[::4] = a[::4]
        L, Rr = sorted_partition(rng, m, es, n)
        lut = rnd(rng, 2 * m, es, 8 * es)
        out = dict(es=es, n=n, alpha=a, seed0=s0, seed1=s1, key=key, maskedX=mx, left=L, right=Rr, lut=lut)
        for p, s in ((0, s0), (1, s1)):
            out[f"eq{p}"] = R.grotto_eq_eval(mx, key, s, p, n)
            out[f"lt{p}"] = R.grotto_eval(mx, key, s, False, p, n)
            out[f"le{p}"] = R.grotto_eval(mx, key, s, True, p, n)
            out[f"mic{p}"] = R.grotto_mic_eval(mx, key, s, p, L, Rr, n)
            e, t = R.grotto_interval_lut_eval(mx, key, s, p, L, Rr, lut, n, 8 * es)
            out[f"lutE{p}"], out[f"lutT{p}"] = e, t
        save(f"grotto_u{8 * es}_n{n}", **out)

    # Grotto full domain (n = 10): reference grottoEqEval / grottoEval(le) at every x.
    es, n, N = 2, 10, 4
    a = rnd(rng, N, es, n)
    s0, s1 = seeds(rng, N), seeds(rng, N)
    key = R.grotto_keygen(a, s0, s1, n)
    dom = 1 << n
    idx = np.repeat(np.arange(N), dom)
    kk = take_elements(key, grotto_regions(n, es), N, idx)
    xs = np.tile(np.arange(dom, dtype=np.uint16), N)
    out = dict(es=es, n=n, alpha=a, seed0=s0, seed1=s1, key=key)
    for p, s in ((0, s0), (1, s1)):
        ss = s.reshape(N, 16)[idx].reshape(-1)
        out[f"eqbits{p}"] = np.packbits(R.grotto_eq_eval(xs, kk, ss, p, n).astype(np.uint8), bitorder="little")
        out[f"lebits{p}"] = np.packbits(R.grotto_eval(xs, kk, ss, True, p, n).astype(np.uint8), bitorder="little")
    save("grotto_all_u16_n10", **out)

    # DCF-based MIC (tests/mic/mic_eval_test_case.h shapes).
    for es, n, bo, N, m in ((4, 32, 32, 32, 4), (1, 8, 8, 32, 3), (8, 64, 64, 16, 4)):
        a = rnd(rng, N, es, n)
        s0, s1 = seeds(rng, N), seeds(rng, N)
        L, Rr = random_intervals(rng, m, es, n)
        key, z = R.dcf_mic_keygen(a, s0, s1, L, Rr, n, bo)
        z0 = rnd(rng, N * m, es, 8 * es)
        z1 = (z.astype(np.uint64) - z0.astype(np.uint64)).astype(DTYPES[es])
        mx = rnd(rng, N, es, 8 * es)
        save(f"dcf_mic_u{8 * es}_n{n}", es=es, n=n, bo=bo, alpha=a, seed0=s0, seed1=s1, left=L, right=Rr, key=key,
             z=z, z0=z0, z1=z1, maskedX=mx, y0=R.dcf_mic_eval(mx, key, z0, s0, 0, L, Rr, n, bo),
             y1=R.dcf_mic_eval(mx, key, z1, s1, 1, L, Rr, n, bo))

    # Spline (tests/spline/spline_eval_test_case.h shapes; BASELINE degree-2 u64).
    for es, m, d, N in ((8, 4, 2, 8), (2, 3, 1, 16), (4, 2, 0, 16)):
        n = bo = 8 * es
        a = rnd(rng, N, es, n)
        s0, s1 = seeds(rng, N), seeds(rng, N)
        L, Rr = sorted_partition(rng, m, es, n)
        coeffs = rnd(rng, m * (d + 1), es, 8 * es)
        key, e, beta = R.spline_keygen(a, s0, s1, coeffs, d, L, Rr, n, bo)
        mx = rnd(rng, N, es, 8 * es)
        e0, b0 = rnd(rng, e.size, es, 8 * es), rnd(rng, beta.size, es, 8 * es)
        e1 = (e.astype(np.uint64) - e0.astype(np.uint64)).astype(DTYPES[es])
        b1 = (beta.astype(np.uint64) - b0.astype(np.uint64)).astype(DTYPES[es])
        save(f"spline_u{8 * es}_m{m}_d{d}", es=es, n=n, bo=bo, d=d, alpha=a, seed0=s0, seed1=s1, left=L, right=Rr,
             coeffs=coeffs, key=key, e=e, beta=beta, e0=e0, e1=e1, b0=b0, b1=b1, maskedX=mx,
             y0=R.spline_eval(mx, key, e0, b0, s0, 0, L, Rr, d, n, bo),
             y1=R.spline_eval(mx, key, e1, b1, s1, 1, L, Rr, d, n, bo))

    # OTTT.
    for es, n, N, lutn in ((1, 8, 16, 2), (2, 10, 8, 1), (4, 3, 16, 3)):
        a = rnd(rng, N, es, n)
        k0 = rng.integers(0, 256, size=N * (1 << n) // 8, dtype=np.uint8)
        k1 = R.ottt_keygen(k0, a, n)
        lut = rnd(rng, (1 << n) * lutn, es, 8 * es)
        mx = rnd(rng, N, es, 8 * es)
        e0, t0 = R.ottt_lut_eval(mx, k0, 0, lut, n)
        e1, t1 = R.ottt_lut_eval(mx, k1, 1, lut, n)
        save(f"ottt_u{8 * es}_n{n}", es=es, n=n, alpha=a, key0=k0, key1=k1, lut=lut, maskedX=mx, e0=e0, t0=t0, e1=e1,
             t1=t1)

    # AES-CTR PRNG (src/cpu/prng.cpp).
    seed = bytes(range(16))
    ctr = (2**64 - 3).to_bytes(8, "little") + (5).to_bytes(8, "little")
    out, ctr_after = R.prng(seed, ctr, 1000)
    save("prng", seed=np.frombuffer(seed, np.uint8), counter=np.frombuffer(ctr, np.uint8), out=out,
         counter_after=np.frombuffer(ctr_after, np.uint8))


if __name__ == "__main__":
    main()
