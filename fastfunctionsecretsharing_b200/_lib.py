"""Loader for the in-tree ``lib/libFastFss.so`` (the C ABI of include/FastFss).

The product path has no fallback: if the library is missing or fails to load, every call
raises. Build it with ``python -m fastfunctionsecretsharing_b200.build``.
"""

from __future__ import annotations

import ctypes
import os
import threading
from ctypes import c_bool, c_int, c_size_t, c_void_p

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libFastFss.so")

_P = c_void_p
_S = c_size_t
_I = c_int

# name -> (restype, argtypes); the prototypes of include/FastFss/**/*.h
SIGNATURES: dict[str, tuple] = {
    # host-side sizes
    "FastFss_dcfKeyZip": (_I, [_P, _S, _P, _S, _S, _S, _S, _S, _S]),
    "FastFss_dcfKeyUnzip": (_I, [_P, _S, _P, _S, _S, _S, _S, _S, _S]),
    "FastFss_dcfGetKeyDataSize": (_I, [_P, _S, _S, _S, _S, _S]),
    "FastFss_dcfGetZippedKeyDataSize": (_I, [_P, _S, _S, _S, _S, _S]),
    "FastFss_dcfGetCacheDataSize": (_I, [_P, _S, _S, _S, _S, _S]),
    "FastFss_dpfKeyZip": (_I, [_P, _S, _P, _S, _S, _S, _S, _S, _S]),
    "FastFss_dpfKeyUnzip": (_I, [_P, _S, _P, _S, _S, _S, _S, _S, _S]),
    "FastFss_dpfGetKeyDataSize": (_I, [_P, _S, _S, _S, _S, _S]),
    "FastFss_dpfGetZippedKeyDataSize": (_I, [_P, _S, _S, _S, _S, _S]),
    "FastFss_dpfGetCacheDataSize": (_I, [_P, _S, _S, _S]),
    "FastFss_grottoKeyZip": (_I, [_P, _S, _P, _S, _S, _S, _S]),
    "FastFss_grottoKeyUnzip": (_I, [_P, _S, _P, _S, _S, _S, _S]),
    "FastFss_grottoGetKeyDataSize": (_I, [_P, _S, _S, _S]),
    "FastFss_grottoGetZippedKeyDataSize": (_I, [_P, _S, _S, _S]),
    "FastFss_grottoGetCacheDataSize": (_I, [_P, _S, _S, _S]),
    "FastFss_dcfMICKeyZip": (_I, [_P, _S, _P, _S, _S, _S, _S, _S]),
    "FastFss_dcfMICKeyUnzip": (_I, [_P, _S, _P, _S, _S, _S, _S, _S]),
    "FastFss_dcfMICGetCacheDataSize": (_I, [_P, _S, _S, _S, _S]),
    "FastFss_dcfMICGetKeyDataSize": (_I, [_P, _S, _S, _S, _S]),
    "FastFss_dcfMICGetZippedKeyDataSize": (_I, [_P, _S, _S, _S, _S]),
    "FastFss_dcfSplineKeyZip": (_I, [_P, _S, _P, _S, _S, _S, _S, _S, _S, _S]),
    "FastFss_dcfSplineKeyUnzip": (_I, [_P, _S, _P, _S, _S, _S, _S, _S, _S, _S]),
    "FastFss_dcfSplineGetCacheDataSize": (_I, [_P, _S, _S, _S, _S, _S, _S]),
    "FastFss_dcfSplineGetKeyDataSize": (_I, [_P, _S, _S, _S, _S, _S, _S]),
    "FastFss_dcfSplineGetZippedKeyDataSize": (_I, [_P, _S, _S, _S, _S, _S, _S]),
    "FastFss_otttGetKeyDataSize": (_I, [_P, _S, _S]),
    # config
    "FastFss_cuda_setGridDim": (_I, [_I]),
    "FastFss_cuda_getGridDim": (_I, []),
    "FastFss_cuda_getFineGrainParallelGridDimThreshold": (_I, []),
    "FastFss_cuda_setFineGrainParallelGridDimThreshold": (_I, [_I]),
    # DCF
    "FastFss_cuda_dcfKeyGen": (_I, [_P, _S, _P, _S, _P, _S, _P, _S, _P, _S, _S, _S, _S, _S, _S, _P]),
    "FastFss_cuda_dcfEval": (_I, [_P, _S, _P, _S, _P, _S, _P, _S, _I, _S, _S, _S, _S, _S, _P, _S, _P]),
    # DPF
    "FastFss_cuda_dpfKeyGen": (_I, [_P, _S, _P, _S, _P, _S, _P, _S, _P, _S, _S, _S, _S, _S, _S, _P]),
    "FastFss_cuda_dpfEval": (_I, [_P, _S, _P, _S, _P, _S, _P, _S, _I, _S, _S, _S, _S, _S, _P, _S, _P]),
    "FastFss_cuda_dpfEvalAll": (_I, [_P, _S, _P, _S, _P, _S, _P, _S, _I, _S, _S, _S, _S, _S, _P, _S, _P]),
    "FastFss_cuda_dpfEvalMulti": (_I, [_P, _S, _P, _S, _P, _S, _P, _S, _I, _P, _S, _S, _S, _S, _S, _S, _P, _S, _P]),
    # Grotto
    "FastFss_cuda_grottoKeyGen": (_I, [_P, _S, _P, _S, _P, _S, _P, _S, _S, _S, _S, _P]),
    "FastFss_cuda_grottoEqEval": (_I, [_P, _S, _P, _S, _P, _S, _P, _S, _I, _S, _S, _S, _P, _S, _P]),
    "FastFss_cuda_grottoEval": (_I, [_P, _S, _P, _S, _P, _S, _P, _S, c_bool, _I, _S, _S, _S, _P, _S, _P]),
    "FastFss_cuda_grottoMICEval": (_I, [_P, _S, _P, _S, _P, _S, _P, _S, _I, _P, _S, _P, _S, _S, _S, _S, _P, _S, _P]),
    "FastFss_cuda_grottoIntervalLutEval": (
        _I, [_P, _S, _P, _S, _P, _S, _P, _S, _P, _S, _I, _P, _S, _P, _S, _P, _S, _S, _S, _S, _S, _P, _S, _P]),
    # DCF MIC
    "FastFss_cuda_dcfMICKeyGen": (_I, [_P, _S, _P, _S, _P, _S, _P, _S, _P, _S, _P, _S, _P, _S, _S, _S, _S, _S, _P]),
    "FastFss_cuda_dcfMICEval": (
        _I, [_P, _S, _P, _S, _P, _S, _P, _S, _P, _S, _I, _P, _S, _P, _S, _S, _S, _S, _S, _P, _S, _P]),
    # spline
    "FastFss_cuda_dcfSplineKeyGen": (
        _I, [_P, _S, _P, _S, _P, _S, _P, _S, _P, _S, _P, _S, _P, _S, _S, _P, _S, _P, _S, _S, _S, _S, _S, _S, _P]),
    "FastFss_cuda_dcfSplineEval": (
        _I, [_P, _S, _P, _S, _P, _S, _P, _S, _P, _S, _P, _S, _I, _P, _S, _P, _S, _S, _S, _S, _S, _S, _S, _P, _S, _P]),
    # OTTT
    "FastFss_cuda_otttKeyGen": (_I, [_P, _S, _P, _S, _S, _S, _S, _P]),
    "FastFss_cuda_otttLutEval": (_I, [_P, _S, _P, _S, _P, _S, _P, _S, _I, _P, _S, _S, _S, _S, _P]),
    # PRNG
    "FastFss_cuda_prngInit": (_P, []),
    "FastFss_cuda_prngRelease": (None, [_P]),
    "FastFss_cuda_prngSetCurrentSeed": (_I, [_P, _P, _P]),
    "FastFss_cuda_prngGetCurrentSeed": (_I, [_P, _P, _P]),
    "FastFss_cuda_prngGen": (_I, [_P, _P, _S, _S, _S, _P]),
}

# Extensions of this library (declared in include/FastFss/b200/*.h).
EXTENSION_SIGNATURES: dict[str, tuple] = {
    "FastFss_b200_smemLookupProbe": (_I, [_P, _S, ctypes.c_uint, _P, _P]),
    "FastFss_b200_smCount": (_I, []),
    "FastFss_b200_stageTimeouts": (_I, [_P]),
    "FastFss_cuda_grottoEqEvalAll": (_I, [_P, _S, _P, _S, _P, _S, _I, _S, _S, _S, _P]),
    "FastFss_cuda_grottoLeEvalAll": (_I, [_P, _S, _P, _S, _P, _S, _I, _S, _S, _S, _P]),
    "FastFss_cuda_grottoIntervalLutEvalFromRows": (
        _I, [_P, _S, _P, _S, _P, _S, _P, _S, _I, _P, _S, _P, _S, _P, _S, _S, _S, _S, _P]),
    "FastFss_cuda_batchEvalNoAlloc": (_I, [_P, _S, _P, _P]),
}

_lock = threading.Lock()
_lib: ctypes.CDLL | None = None


def load() -> ctypes.CDLL:
    """Returns the loaded library; raises if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m fastfunctionsecretsharing_b200.build` "
                    "(this package has no CPU fallback)")
            lib = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in {**SIGNATURES, **EXTENSION_SIGNATURES}.items():
                fn = getattr(lib, name, None)
                if fn is None:
                    continue
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def fn(name: str):
    f = getattr(load(), name, None)
    if f is None:
        raise RuntimeError(f"{name} is not exported by {LIB_PATH}")
    return f
