"""ctypes front end of the test oracle (TEST INFRASTRUCTURE ONLY).

Two CPU back ends share one numpy-level interface:

* ``Oracle``  — the plain-C restatement in ``fss_oracle.c`` (``liboracle.so``).
* ``RefCpu``  — the reference's own CPU library (``FastFss_cpu_*`` from src/cpu/*.cpp),
  compiled from the reference sources into ``_ref/libfastfss_ref.so`` by ``make ref``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import
this module; the product library never does.

Every method takes numpy arrays (ring elements as uint8/16/32/64, seeds and keys as uint8)
and returns freshly allocated numpy outputs. Element size comes from the element dtype.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import c_bool, c_int, c_size_t, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libfastfss_ref.so")

DTYPES = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}


def _ptr(a):
    if a is None:
        return None
    return c_void_p(a.ctypes.data)


def _es(a):
    return np.dtype(a.dtype).itemsize


def build(ref: bool = False) -> None:
    """Compile the restatement (and, with ``ref``, the reference CPU library)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


# ----------------------------------------------------------------------------------------
# key / cache sizes (restated from src/impl/*.h so the oracle does not need the product)
# ----------------------------------------------------------------------------------------

def dcf_key_size(n, bo, g, es, N):
    return N * (16 * n + es * n * g + es + es + es * g)


def dpf_key_size(n, bo, g, es, N):
    return N * (16 * n + es + es + es * g)


def grotto_key_size(n, es, N):
    return N * (16 * (n - 6) + 8 + 2 * es)


def spline_key_size(n, bo, m, d, es, N):
    return dcf_key_size(n, bo, m * (d + 1), es, N)


def spline_cache_size(n, bo, m, d, es, N):
    g = m * (d + 1)
    return N * 16 * n + N * es * n * g + N * es * (2 * g + d + 1)


def ottt_key_size(n, N):
    return N * (1 << n) // 8


class _Base:
    lib: ctypes.CDLL

    # subclasses implement the raw calls; the numpy API lives here

    def dcf_keygen(self, alpha, beta, seed0, seed1, n, bo, g):
        es, N = _es(alpha), alpha.size
        key = np.zeros(dcf_key_size(n, bo, g, es, N), np.uint8)
        self._dcf_keygen(key, alpha, beta, seed0, seed1, n, bo, g, es, N)
        return key

    def dcf_eval(self, maskedX, key, seed, party, n, bo, g):
        es, N = _es(maskedX), maskedX.size
        out = np.zeros(N * g, maskedX.dtype)
        self._dcf_eval(out, maskedX, key, seed, party, n, bo, g, es, N)
        return out

    def dpf_keygen(self, alpha, beta, seed0, seed1, n, bo, g):
        es, N = _es(alpha), alpha.size
        key = np.zeros(dpf_key_size(n, bo, g, es, N), np.uint8)
        self._dpf_keygen(key, alpha, beta, seed0, seed1, n, bo, g, es, N)
        return key

    def dpf_eval(self, maskedX, key, seed, party, n, bo, g):
        es, N = _es(maskedX), maskedX.size
        out = np.zeros(N * g, maskedX.dtype)
        self._dpf_eval(out, maskedX, key, seed, party, n, bo, g, es, N)
        return out

    def dpf_eval_all(self, maskedX, key, seed, party, n, bo, g):
        es, N = _es(maskedX), maskedX.size
        out = np.zeros(N * (1 << n) * g, maskedX.dtype)
        self._dpf_eval_all(out, maskedX, key, seed, party, n, bo, g, es, N)
        return out

    def dpf_eval_multi(self, maskedX, key, seed, party, point, n, bo, g):
        es, N = _es(maskedX), maskedX.size
        out = np.zeros(N * point.size * g, maskedX.dtype)
        self._dpf_eval_multi(out, maskedX, key, seed, party, point, n, bo, g, es, N)
        return out

    def grotto_keygen(self, alpha, seed0, seed1, n):
        es, N = _es(alpha), alpha.size
        key = np.zeros(grotto_key_size(n, es, N), np.uint8)
        self._grotto_keygen(key, alpha, seed0, seed1, n, es, N)
        return key

    def grotto_eq_eval(self, maskedX, key, seed, party, n):
        es, N = _es(maskedX), maskedX.size
        out = np.zeros(N, maskedX.dtype)
        self._grotto_eq_eval(out, maskedX, key, seed, party, n, es, N)
        return out

    def grotto_eval(self, maskedX, key, seed, equal_bound, party, n):
        es, N = _es(maskedX), maskedX.size
        out = np.zeros(N, maskedX.dtype)
        self._grotto_eval(out, maskedX, key, seed, equal_bound, party, n, es, N)
        return out

    def grotto_mic_eval(self, maskedX, key, seed, party, left, right, n):
        es, N = _es(maskedX), maskedX.size
        out = np.zeros(N * left.size, maskedX.dtype)
        self._grotto_mic_eval(out, maskedX, key, seed, party, left, right, n, es, N)
        return out

    def grotto_interval_lut_eval(self, maskedX, key, seed, party, left, right, lut, n, bo):
        es, N = _es(maskedX), maskedX.size
        m = left.size
        lut_num = lut.size // m if m else 0
        outE = np.zeros(N, maskedX.dtype)
        outT = np.zeros(N * lut_num, maskedX.dtype)
        self._grotto_lut_eval(outE, outT, maskedX, key, seed, party, left, right, lut, n, bo, es, N)
        return outE, outT

    def dcf_mic_keygen(self, alpha, seed0, seed1, left, right, n, bo):
        es, N = _es(alpha), alpha.size
        key = np.zeros(dcf_key_size(n, bo, 1, es, N), np.uint8)
        z = np.zeros(N * left.size, alpha.dtype)
        self._dcf_mic_keygen(key, z, alpha, seed0, seed1, left, right, n, bo, es, N)
        return key, z

    def dcf_mic_eval(self, maskedX, key, z, seed, party, left, right, n, bo):
        es, N = _es(maskedX), maskedX.size
        out = np.zeros(N * left.size, maskedX.dtype)
        self._dcf_mic_eval(out, maskedX, key, z, seed, party, left, right, n, bo, es, N)
        return out

    def spline_keygen(self, alpha, seed0, seed1, coeffs, degree, left, right, n, bo):
        es, N = _es(alpha), alpha.size
        m = left.size
        g = m * (degree + 1)
        key = np.zeros(spline_key_size(n, bo, m, degree, es, N), np.uint8)
        e = np.zeros(N * g, alpha.dtype)
        beta = np.zeros(N * g, alpha.dtype)
        self._spline_keygen(key, e, beta, alpha, seed0, seed1, coeffs, degree, left, right, n, bo, es, N)
        return key, e, beta

    def spline_eval(self, maskedX, key, e, beta, seed, party, left, right, degree, n, bo):
        es, N = _es(maskedX), maskedX.size
        out = np.zeros(N, maskedX.dtype)
        self._spline_eval(out, maskedX, key, e, beta, seed, party, left, right, degree, n, bo, es, N)
        return out

    def ottt_keygen(self, key_in, alpha, n):
        es, N = _es(alpha), alpha.size
        key = key_in.copy()
        self._ottt_keygen(key, alpha, n, es, N)
        return key

    def ottt_lut_eval(self, maskedX, key, party, lut, n):
        es, N = _es(maskedX), maskedX.size
        lut_num = lut.size // (1 << n)
        outE = np.zeros(N, maskedX.dtype)
        outT = np.zeros(N * lut_num, maskedX.dtype)
        self._ottt_lut_eval(outE, outT, maskedX, key, party, lut, n, es, N)
        return outE, outT


class Oracle(_Base):
    """The C restatement (fss_oracle.c)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build(ref=False)
        self.lib = ctypes.CDLL(path)
        self.lib.oracle_set_num_threads.argtypes = [c_int]

    def set_threads(self, n: int) -> None:
        self.lib.oracle_set_num_threads(n)

    def aes128(self, key16: bytes, block16: bytes) -> bytes:
        out = ctypes.create_string_buffer(16)
        self.lib.oracle_aes128_encrypt(key16, block16, out)
        return out.raw

    def prng(self, seed16: bytes, counter16: bytes, nbytes: int):
        ctr = ctypes.create_string_buffer(counter16, 16)
        out = np.zeros(nbytes, np.uint8)
        self.lib.oracle_prng_gen(seed16, ctr, _ptr(out), c_size_t(nbytes))
        return out, ctr.raw

    def _dcf_keygen(self, key, alpha, beta, s0, s1, n, bo, g, es, N):
        self.lib.oracle_dcfKeyGen(_ptr(key), _ptr(alpha), _ptr(beta), _ptr(s0), _ptr(s1), c_size_t(n),
                                  c_size_t(bo), c_size_t(g), c_size_t(es), c_size_t(N))

    def _dcf_eval(self, out, x, key, seed, party, n, bo, g, es, N):
        self.lib.oracle_dcfEval(_ptr(out), _ptr(x), _ptr(key), _ptr(seed), c_int(party), c_size_t(n),
                                c_size_t(bo), c_size_t(g), c_size_t(es), c_size_t(N))

    def _dpf_keygen(self, key, alpha, beta, s0, s1, n, bo, g, es, N):
        self.lib.oracle_dpfKeyGen(_ptr(key), _ptr(alpha), _ptr(beta), _ptr(s0), _ptr(s1), c_size_t(n),
                                  c_size_t(bo), c_size_t(g), c_size_t(es), c_size_t(N))

    def _dpf_eval(self, out, x, key, seed, party, n, bo, g, es, N):
        self.lib.oracle_dpfEval(_ptr(out), _ptr(x), _ptr(key), _ptr(seed), c_int(party), c_size_t(n),
                                c_size_t(bo), c_size_t(g), c_size_t(es), c_size_t(N))

    def _dpf_eval_all(self, out, x, key, seed, party, n, bo, g, es, N):
        self.lib.oracle_dpfEvalAll(_ptr(out), _ptr(x), _ptr(key), _ptr(seed), c_int(party), c_size_t(n),
                                   c_size_t(bo), c_size_t(g), c_size_t(es), c_size_t(N))

    def _dpf_eval_multi(self, out, x, key, seed, party, point, n, bo, g, es, N):
        self.lib.oracle_dpfEvalMulti(_ptr(out), _ptr(x), _ptr(key), _ptr(seed), c_int(party), _ptr(point),
                                     c_size_t(point.size), c_size_t(n), c_size_t(bo), c_size_t(g), c_size_t(es),
                                     c_size_t(N))

    def _grotto_keygen(self, key, alpha, s0, s1, n, es, N):
        self.lib.oracle_grottoKeyGen(_ptr(key), _ptr(alpha), _ptr(s0), _ptr(s1), c_size_t(n), c_size_t(es),
                                     c_size_t(N))

    def _grotto_eq_eval(self, out, x, key, seed, party, n, es, N):
        self.lib.oracle_grottoEqEval(_ptr(out), _ptr(x), _ptr(key), _ptr(seed), c_int(party), c_size_t(n),
                                     c_size_t(es), c_size_t(N))

    def _grotto_eval(self, out, x, key, seed, eb, party, n, es, N):
        self.lib.oracle_grottoEval(_ptr(out), _ptr(x), _ptr(key), _ptr(seed), c_int(int(eb)), c_int(party),
                                   c_size_t(n), c_size_t(es), c_size_t(N))

    def _grotto_mic_eval(self, out, x, key, seed, party, left, right, n, es, N):
        self.lib.oracle_grottoMICEval(_ptr(out), _ptr(x), _ptr(key), _ptr(seed), c_int(party), _ptr(left),
                                      _ptr(right), c_size_t(left.size), c_size_t(n), c_size_t(es), c_size_t(N))

    def _grotto_lut_eval(self, outE, outT, x, key, seed, party, left, right, lut, n, bo, es, N):
        m = left.size
        self.lib.oracle_grottoIntervalLutEval(_ptr(outE), _ptr(outT), _ptr(x), _ptr(key), _ptr(seed), c_int(party),
                                              _ptr(left), _ptr(right), _ptr(lut), c_size_t(lut.size // m if m else 0),
                                              c_size_t(m), c_size_t(n), c_size_t(es), c_size_t(N))

    def grotto_eq_eval_all(self, key, seed, party, n, es, N):
        out = np.zeros(N * (1 << n) // 8, np.uint8)
        self.lib.oracle_grottoEqEvalAll(_ptr(out), _ptr(key), _ptr(seed), c_int(party), c_size_t(n), c_size_t(es),
                                        c_size_t(N))
        return out

    def grotto_le_eval_all(self, key, seed, party, n, es, N):
        out = np.zeros(N * (1 << n) // 8, np.uint8)
        self.lib.oracle_grottoLeEvalAll(_ptr(out), _ptr(key), _ptr(seed), c_int(party), c_size_t(n), c_size_t(es),
                                        c_size_t(N))
        return out

    def _dcf_mic_keygen(self, key, z, alpha, s0, s1, left, right, n, bo, es, N):
        self.lib.oracle_dcfMICKeyGen(_ptr(key), _ptr(z), _ptr(alpha), _ptr(s0), _ptr(s1), _ptr(left), _ptr(right),
                                     c_size_t(left.size), c_size_t(n), c_size_t(bo), c_size_t(es), c_size_t(N))

    def _dcf_mic_eval(self, out, x, key, z, seed, party, left, right, n, bo, es, N):
        self.lib.oracle_dcfMICEval(_ptr(out), _ptr(x), _ptr(key), _ptr(z), _ptr(seed), c_int(party), _ptr(left),
                                   _ptr(right), c_size_t(left.size), c_size_t(n), c_size_t(bo), c_size_t(es),
                                   c_size_t(N))

    def _spline_keygen(self, key, e, beta, alpha, s0, s1, coeffs, d, left, right, n, bo, es, N):
        self.lib.oracle_dcfSplineKeyGen(_ptr(key), _ptr(e), _ptr(beta), _ptr(alpha), _ptr(s0), _ptr(s1),
                                        _ptr(coeffs), c_size_t(d), _ptr(left), _ptr(right), c_size_t(left.size),
                                        c_size_t(n), c_size_t(bo), c_size_t(es), c_size_t(N))

    def _spline_eval(self, out, x, key, e, beta, seed, party, left, right, d, n, bo, es, N):
        self.lib.oracle_dcfSplineEval(_ptr(out), _ptr(x), _ptr(key), _ptr(e), _ptr(beta), _ptr(seed), c_int(party),
                                      _ptr(left), _ptr(right), c_size_t(left.size), c_size_t(d), c_size_t(n),
                                      c_size_t(bo), c_size_t(es), c_size_t(N))

    def _ottt_keygen(self, key, alpha, n, es, N):
        self.lib.oracle_otttKeyGen(_ptr(key), _ptr(alpha), c_size_t(n), c_size_t(es), c_size_t(N))

    def _ottt_lut_eval(self, outE, outT, x, key, party, lut, n, es, N):
        self.lib.oracle_otttLutEval(_ptr(outE), _ptr(outT), _ptr(x), _ptr(key), c_int(party), _ptr(lut),
                                    c_size_t(lut.size // (1 << n)), c_size_t(n), c_size_t(es), c_size_t(N))


class RefError(RuntimeError):
    pass


def _chk(rc, what):
    if rc != 0:
        raise RefError(f"{what} returned {rc}")


def _nb(a):
    return c_size_t(0 if a is None else a.nbytes)


class RefCpu(_Base):
    """The reference's own CPU library (FastFss_cpu_*), built from its sources."""

    def __init__(self, path: str = REF_SO):
        self.lib = ctypes.CDLL(path)
        self.lib.FastFss_cpu_prngInit.restype = c_void_p

    @staticmethod
    def available(path: str = REF_SO) -> bool:
        return os.path.exists(path)

    def set_threads(self, n: int) -> None:
        self.lib.FastFss_cpu_setNumThreads(c_int(n))

    def prng(self, seed16: bytes, counter16: bytes, nbytes: int):
        h = c_void_p(self.lib.FastFss_cpu_prngInit())
        try:
            _chk(self.lib.FastFss_cpu_prngSetCurrentSeed(h, seed16, counter16), "prngSetCurrentSeed")
            out = np.zeros(nbytes, np.uint8)
            _chk(self.lib.FastFss_cpu_prngGen(h, _ptr(out), c_size_t(8), c_size_t(1), c_size_t(nbytes)), "prngGen")
            s = ctypes.create_string_buffer(16)
            c = ctypes.create_string_buffer(16)
            _chk(self.lib.FastFss_cpu_prngGetCurrentSeed(h, s, c), "prngGetCurrentSeed")
            return out, c.raw
        finally:
            self.lib.FastFss_cpu_prngRelease(h)

    def _dcf_keygen(self, key, alpha, beta, s0, s1, n, bo, g, es, N):
        _chk(self.lib.FastFss_cpu_dcfKeyGen(_ptr(key), _nb(key), _ptr(alpha), _nb(alpha), _ptr(beta), _nb(beta),
                                            _ptr(s0), _nb(s0), _ptr(s1), _nb(s1), c_size_t(n), c_size_t(bo),
                                            c_size_t(g), c_size_t(es), c_size_t(N)), "dcfKeyGen")

    def _dcf_eval(self, out, x, key, seed, party, n, bo, g, es, N):
        _chk(self.lib.FastFss_cpu_dcfEval(_ptr(out), _nb(out), _ptr(x), _nb(x), _ptr(key), _nb(key), _ptr(seed),
                                          _nb(seed), c_int(party), c_size_t(n), c_size_t(bo), c_size_t(g),
                                          c_size_t(es), c_size_t(N), None, c_size_t(0)), "dcfEval")

    def _dpf_keygen(self, key, alpha, beta, s0, s1, n, bo, g, es, N):
        _chk(self.lib.FastFss_cpu_dpfKeyGen(_ptr(key), _nb(key), _ptr(alpha), _nb(alpha), _ptr(beta), _nb(beta),
                                            _ptr(s0), _nb(s0), _ptr(s1), _nb(s1), c_size_t(n), c_size_t(bo),
                                            c_size_t(g), c_size_t(es), c_size_t(N)), "dpfKeyGen")

    def _dpf_eval(self, out, x, key, seed, party, n, bo, g, es, N):
        _chk(self.lib.FastFss_cpu_dpfEval(_ptr(out), _nb(out), _ptr(x), _nb(x), _ptr(key), _nb(key), _ptr(seed),
                                          _nb(seed), c_int(party), c_size_t(n), c_size_t(bo), c_size_t(g),
                                          c_size_t(es), c_size_t(N), None, c_size_t(0)), "dpfEval")

    def _dpf_eval_all(self, out, x, key, seed, party, n, bo, g, es, N):
        _chk(self.lib.FastFss_cpu_dpfEvalAll(_ptr(out), _nb(out), _ptr(x), _nb(x), _ptr(key), _nb(key), _ptr(seed),
                                             _nb(seed), c_int(party), c_size_t(n), c_size_t(bo), c_size_t(g),
                                             c_size_t(es), c_size_t(N), None, c_size_t(0)), "dpfEvalAll")

    def _dpf_eval_multi(self, out, x, key, seed, party, point, n, bo, g, es, N):
        _chk(self.lib.FastFss_cpu_dpfEvalMulti(_ptr(out), _nb(out), _ptr(x), _nb(x), _ptr(key), _nb(key), _ptr(seed),
                                               _nb(seed), c_int(party), _ptr(point), _nb(point), c_size_t(n),
                                               c_size_t(bo), c_size_t(g), c_size_t(es), c_size_t(N), None,
                                               c_size_t(0)), "dpfEvalMulti")

    def _grotto_keygen(self, key, alpha, s0, s1, n, es, N):
        _chk(self.lib.FastFss_cpu_grottoKeyGen(_ptr(key), _nb(key), _ptr(alpha), _nb(alpha), _ptr(s0), _nb(s0),
                                               _ptr(s1), _nb(s1), c_size_t(n), c_size_t(es), c_size_t(N)),
             "grottoKeyGen")

    def _grotto_eq_eval(self, out, x, key, seed, party, n, es, N):
        _chk(self.lib.FastFss_cpu_grottoEqEval(_ptr(out), _nb(out), _ptr(x), _nb(x), _ptr(key), _nb(key), _ptr(seed),
                                               _nb(seed), c_int(party), c_size_t(n), c_size_t(es), c_size_t(N), None,
                                               c_size_t(0)), "grottoEqEval")

    def _grotto_eval(self, out, x, key, seed, eb, party, n, es, N):
        _chk(self.lib.FastFss_cpu_grottoEval(_ptr(out), _nb(out), _ptr(x), _nb(x), _ptr(key), _nb(key), _ptr(seed),
                                             _nb(seed), c_bool(bool(eb)), c_int(party), c_size_t(n), c_size_t(es),
                                             c_size_t(N), None, c_size_t(0)), "grottoEval")

    def _grotto_mic_eval(self, out, x, key, seed, party, left, right, n, es, N):
        _chk(self.lib.FastFss_cpu_grottoMICEval(_ptr(out), _nb(out), _ptr(x), _nb(x), _ptr(key), _nb(key),
                                                _ptr(seed), _nb(seed), c_int(party), _ptr(left), _nb(left),
                                                _ptr(right), _nb(right), c_size_t(n), c_size_t(es), c_size_t(N), None,
                                                c_size_t(0)), "grottoMICEval")

    def _grotto_lut_eval(self, outE, outT, x, key, seed, party, left, right, lut, n, bo, es, N):
        _chk(self.lib.FastFss_cpu_grottoIntervalLutEval(_ptr(outE), _nb(outE), _ptr(outT), _nb(outT), _ptr(x), _nb(x),
                                                        _ptr(key), _nb(key), _ptr(seed), _nb(seed), c_int(party),
                                                        _ptr(left), _nb(left), _ptr(right), _nb(right), _ptr(lut),
                                                        _nb(lut), c_size_t(n), c_size_t(bo), c_size_t(es), c_size_t(N),
                                                        None, c_size_t(0)), "grottoIntervalLutEval")

    def _dcf_mic_keygen(self, key, z, alpha, s0, s1, left, right, n, bo, es, N):
        _chk(self.lib.FastFss_cpu_dcfMICKeyGen(_ptr(key), _nb(key), _ptr(z), _nb(z), _ptr(alpha), _nb(alpha),
                                               _ptr(s0), _nb(s0), _ptr(s1), _nb(s1), _ptr(left), _nb(left),
                                               _ptr(right), _nb(right), c_size_t(n), c_size_t(bo), c_size_t(es),
                                               c_size_t(N)), "dcfMICKeyGen")

    def _dcf_mic_eval(self, out, x, key, z, seed, party, left, right, n, bo, es, N):
        _chk(self.lib.FastFss_cpu_dcfMICEval(_ptr(out), _nb(out), _ptr(x), _nb(x), _ptr(key), _nb(key), _ptr(z),
                                             _nb(z), _ptr(seed), _nb(seed), c_int(party), _ptr(left), _nb(left),
                                             _ptr(right), _nb(right), c_size_t(n), c_size_t(bo), c_size_t(es),
                                             c_size_t(N), None, c_size_t(0)), "dcfMICEval")

    def _spline_keygen(self, key, e, beta, alpha, s0, s1, coeffs, d, left, right, n, bo, es, N):
        _chk(self.lib.FastFss_cpu_dcfSplineKeyGen(_ptr(key), _nb(key), _ptr(e), _nb(e), _ptr(beta), _nb(beta),
                                                  _ptr(alpha), _nb(alpha), _ptr(s0), _nb(s0), _ptr(s1), _nb(s1),
                                                  _ptr(coeffs), _nb(coeffs), c_size_t(d), _ptr(left), _nb(left),
                                                  _ptr(right), _nb(right), c_size_t(left.size), c_size_t(n),
                                                  c_size_t(bo), c_size_t(es), c_size_t(N)), "dcfSplineKeyGen")

    def _spline_eval(self, out, x, key, e, beta, seed, party, left, right, d, n, bo, es, N):
        m = left.size
        cache = np.zeros(spline_cache_size(n, bo, m, d, es, N), np.uint8)
        _chk(self.lib.FastFss_cpu_dcfSplineEval(_ptr(out), _nb(out), _ptr(x), _nb(x), _ptr(key), _nb(key), _ptr(e),
                                                _nb(e), _ptr(beta), _nb(beta), _ptr(seed), _nb(seed), c_int(party),
                                                _ptr(left), _nb(left), _ptr(right), _nb(right), c_size_t(m),
                                                c_size_t(d), c_size_t(n), c_size_t(bo), c_size_t(es), c_size_t(N),
                                                _ptr(cache), _nb(cache)), "dcfSplineEval")

    def _ottt_keygen(self, key, alpha, n, es, N):
        _chk(self.lib.FastFss_cpu_otttKeyGen(_ptr(key), _nb(key), _ptr(alpha), _nb(alpha), c_size_t(n), c_size_t(es),
                                             c_size_t(N)), "otttKeyGen")

    def _ottt_lut_eval(self, outE, outT, x, key, party, lut, n, es, N):
        _chk(self.lib.FastFss_cpu_otttLutEval(_ptr(outE), _nb(outE), _ptr(outT), _nb(outT), _ptr(x), _nb(x),
                                              _ptr(key), _nb(key), c_int(party), _ptr(lut), _nb(lut), c_size_t(n),
                                              c_size_t(es), c_size_t(N)), "otttLutEval")
