"""Seeded input generators and key-layout helpers shared by the tests (no GPU needed)."""

from __future__ import annotations

import numpy as np

DTYPES = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}


def rnd(rng: np.random.Generator, N: int, es: int, bits: int) -> np.ndarray:
    """N uniform ring elements of es bytes, reduced to `bits` bits."""
    v = rng.integers(0, 2**63, size=N, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, size=N, dtype=np.uint64)
    if bits < 64:
        v &= np.uint64((1 << bits) - 1)
    return v.astype(DTYPES[es])


def seeds(rng: np.random.Generator, N: int) -> np.ndarray:
    return rng.integers(0, 256, size=N * 16, dtype=np.uint8)


def maxval(es: int, bits: int):
    return DTYPES[es]((1 << bits) - 1)


def sorted_partition(rng, m: int, es: int, n: int):
    """m intervals [L_i, R_i] covering [0, 2^n) with distinct sorted left endpoints, L_0 = 0
    (the shape the reference's spline/LUT tests use, tests/common/nbit_signed.hpp:136)."""
    dom = 1 << n
    m = min(m, dom)
    cuts: set[int] = set()
    while len(cuts) < m - 1:
        c = int(rng.integers(0, 2**63, dtype=np.uint64)) * 2 + int(rng.integers(0, 2))
        c %= dom
        if c != 0:
            cuts.add(c)
    L = [0] + sorted(cuts)
    R = [v - 1 for v in L[1:]] + [dom - 1]
    return np.array(L, dtype=np.uint64).astype(DTYPES[es]), np.array(R, dtype=np.uint64).astype(DTYPES[es])


def random_intervals(rng, m: int, es: int, n: int):
    """m independent intervals [L, R] with L <= R < 2^n (not a partition)."""
    a = rnd(rng, m, es, n).astype(np.uint64)
    b = rnd(rng, m, es, n).astype(np.uint64)
    return np.minimum(a, b).astype(DTYPES[es]), np.maximum(a, b).astype(DTYPES[es])


def touching_intervals(rng, m: int, es: int, n: int):
    """m intervals [b_q, b_{q+1} - 1] between sorted distinct boundaries (each touches the next,
    but the last does not wrap round to the first)."""
    dom = 1 << n
    b: set[int] = set()
    while len(b) < m + 1:
        b.add(int(rnd(rng, 1, 8, n)[0]) % dom)
    bs = sorted(b)
    L = np.array(bs[:-1], dtype=np.uint64).astype(DTYPES[es])
    R = np.array([(v - 1) % dom for v in bs[1:]], dtype=np.uint64).astype(DTYPES[es])
    return L, R


def take_elements(key: np.ndarray, regions: list[int], N: int, idx: np.ndarray) -> np.ndarray:
    """Rebuilds a key buffer holding elements `idx` of a key whose layout is a sequence of
    element-major regions with the given per-element byte strides."""
    out = []
    off = 0
    for stride in regions:
        reg = key[off:off + N * stride].reshape(N, stride)
        out.append(reg[idx].reshape(-1))
        off += N * stride
    return np.concatenate(out)


def grotto_regions(n: int, es: int) -> list[int]:
    return [16 * (n - 6), 8, 2 * es]


def dcf_regions(n: int, g: int, es: int) -> list[int]:
    return [16 * n, es * (n * g + 2 + g)]


def dpf_regions(n: int, g: int, es: int) -> list[int]:
    return [16 * n, es * (2 + g)]
