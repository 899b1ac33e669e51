"""FastFss for B200: the function-secret-sharing hot path as sm_100a CUDA kernels.

This module is the Python face of ``lib/libFastFss.so``, which exports the reference's
``include/FastFss`` C ABI. The functions below mirror the torch extension of the reference
(``pyFastFss``, lib/torch_extension/pyFastFss/csrc/bind_*.cpp): same names, argument order and
meaning; outputs are resized in place and returned; a non-zero C-ABI status raises
``RuntimeError("FastFss_cuda_<op> failed : <code>")``.

Tensors must be contiguous CUDA tensors (ring elements in an 8/16/32/64-bit integer dtype,
keys and seeds ``torch.uint8``). Work is queued on the current torch CUDA stream. There is no
CPU path: a CPU tensor raises ``ValueError``.
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib

__all__ = [
    "mod", "dtype", "logical_shape", "logical_numel",
    "dcf_get_key_data_size", "dcf_key_gen", "dcf_eval",
    "dpf_get_key_data_size", "dpf_key_gen", "dpf_eval", "dpf_eval_all", "dpf_multi_eval",
    "grotto_get_key_data_size", "grotto_key_gen", "grotto_eq_eval", "grotto_eval", "grotto_mic_eval",
    "grotto_interval_lut_eval", "grotto_eq_eval_all", "grotto_le_eval_all", "grotto_interval_lut_eval_from_rows",
    "dcf_mic_get_key_data_size", "dcf_mic_key_gen", "dcf_mic_eval",
    "spline_get_key_data_size", "spline_key_gen", "spline_eval",
    "ottt_get_key_data_size", "ottt_key_gen", "ottt_lut_eval",
    "set_grid_dim", "get_grid_dim", "set_fine_grain_parallel_grid_dim_threshold",
    "get_fine_grain_parallel_grid_dim_threshold", "Prng",
]


# ------------------------------------------------------------------------------------
# helpers
# ------------------------------------------------------------------------------------

def mod(x: torch.Tensor, bit_width: int, *, out: torch.Tensor | None = None) -> torch.Tensor:
    """x mod 2^bit_width (lib/torch_extension/pyFastFss/__init__.py:10-38, <= 64 bits)."""
    if out is None:
        out = torch.empty_like(x)
    if x.element_size() * 8 == bit_width:
        return out.copy_(x)
    return torch.bitwise_and(x, (1 << bit_width) - 1, out=out)


def dtype(bit_width: int) -> torch.dtype:
    """Smallest signed integer dtype holding bit_width bits (pyFastFss/__init__.py:41-51)."""
    assert 0 < bit_width <= 64
    if bit_width <= 8:
        return torch.int8
    if bit_width <= 16:
        return torch.int16
    if bit_width <= 32:
        return torch.int32
    return torch.int64


def _wide_limb_num(bit_width: int) -> int:
    return 1 if bit_width <= 64 else (bit_width + 63) // 64


def logical_shape(x: torch.Tensor, bit_width: int) -> torch.Size:
    """Shape of the ring elements held by x (pyFastFss/__init__.py:52-61): x.shape up to 64 bits;
    wider rings are int64 tensors whose last dimension holds the 64-bit limbs (the kernels of this
    library evaluate rings of up to 64 bits)."""
    if bit_width <= 64:
        return x.shape
    if x.dtype != torch.int64:
        raise ValueError("wideint tensors must use torch.int64 dtype")
    if x.ndim < 1 or x.shape[-1] != _wide_limb_num(bit_width):
        raise ValueError("wideint tensor last dimension must equal limb count")
    return x.shape[:-1]


def logical_numel(x: torch.Tensor, bit_width: int) -> int:
    """Number of ring elements held by x (pyFastFss/__init__.py:63-72)."""
    n = 1
    for dim in logical_shape(x, bit_width):
        n *= dim
    return n


def _nbytes(t: torch.Tensor | None) -> int:
    return 0 if t is None else t.numel() * t.element_size()


def _ptr(t: torch.Tensor | None):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _cuda(*ts: torch.Tensor | None) -> torch.device:
    dev = None
    for t in ts:
        if t is None:
            continue
        if not t.is_contiguous():
            raise ValueError("FastFss tensors must be contiguous")
        if t.device.type != "cuda":
            raise ValueError("device not supported: FastFss-B200 runs on CUDA tensors only")
        if dev is None:
            dev = t.device
        elif t.device != dev:
            raise ValueError("all tensors must be on the same CUDA device")
    return dev


class _Stream:
    """Pointer to the current torch stream handle, as the C ABI expects (cudaStream_t*)."""

    def __init__(self, device: torch.device):
        self.handle = ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)

    @property
    def ptr(self):
        return ctypes.byref(self.handle)


def _check(name: str, rc: int) -> None:
    if rc != 0:
        raise RuntimeError(f"{name} failed : {rc}")


def _size_query(name: str, *args) -> int:
    out = ctypes.c_size_t(0)
    _check(name, _lib.fn(name)(ctypes.byref(out), *args))
    return out.value


# ------------------------------------------------------------------------------------
# DCF (bind_dcf.cpp)
# ------------------------------------------------------------------------------------

def dcf_get_key_data_size(bitWidthIn, bitWidthOut, groupSize, elementSize, elementNum) -> int:
    return _size_query("FastFss_dcfGetKeyDataSize", bitWidthIn, bitWidthOut, groupSize, elementSize, elementNum)


def dcf_key_gen(keyOut, alpha, beta, seed0, seed1, bitWidthIn, bitWidthOut, groupSize):
    dev = _cuda(keyOut, alpha, beta, seed0, seed1)
    es, N = alpha.element_size(), alpha.numel()
    keyOut.resize_(dcf_get_key_data_size(bitWidthIn, bitWidthOut, groupSize, es, N))
    st = _Stream(dev)
    _check("FastFss_cuda_dcfKeyGen", _lib.fn("FastFss_cuda_dcfKeyGen")(
        _ptr(keyOut), _nbytes(keyOut), _ptr(alpha), _nbytes(alpha), _ptr(beta), _nbytes(beta), _ptr(seed0),
        _nbytes(seed0), _ptr(seed1), _nbytes(seed1), bitWidthIn, bitWidthOut, groupSize, es, N, st.ptr))
    return keyOut


def dcf_eval(sharedOut, maskedX, key, seed, partyId, bitWidthIn, bitWidthOut, groupSize):
    dev = _cuda(sharedOut, maskedX, key, seed)
    es, N = maskedX.element_size(), maskedX.numel()
    sharedOut.resize_(list(maskedX.shape) + [groupSize])
    st = _Stream(dev)
    _check("FastFss_cuda_dcfEval", _lib.fn("FastFss_cuda_dcfEval")(
        _ptr(sharedOut), _nbytes(sharedOut), _ptr(maskedX), _nbytes(maskedX), _ptr(key), _nbytes(key), _ptr(seed),
        _nbytes(seed), partyId, bitWidthIn, bitWidthOut, groupSize, es, N, None, 0, st.ptr))
    return sharedOut


# ------------------------------------------------------------------------------------
# DPF (bind_dpf.cpp)
# ------------------------------------------------------------------------------------

def dpf_get_key_data_size(bitWidthIn, bitWidthOut, groupSize, elementSize, elementNum) -> int:
    return _size_query("FastFss_dpfGetKeyDataSize", bitWidthIn, bitWidthOut, groupSize, elementSize, elementNum)


def dpf_key_gen(keyOut, alpha, beta, seed0, seed1, bitWidthIn, bitWidthOut, groupSize):
    dev = _cuda(keyOut, alpha, beta, seed0, seed1)
    es, N = alpha.element_size(), alpha.numel()
    keyOut.resize_(dpf_get_key_data_size(bitWidthIn, bitWidthOut, groupSize, es, N))
    st = _Stream(dev)
    _check("FastFss_cuda_dpfKeyGen", _lib.fn("FastFss_cuda_dpfKeyGen")(
        _ptr(keyOut), _nbytes(keyOut), _ptr(alpha), _nbytes(alpha), _ptr(beta), _nbytes(beta), _ptr(seed0),
        _nbytes(seed0), _ptr(seed1), _nbytes(seed1), bitWidthIn, bitWidthOut, groupSize, es, N, st.ptr))
    return keyOut


def _dpf_eval_common(op, sharedOut, out_shape, maskedX, key, seed, partyId, bitWidthIn, bitWidthOut, groupSize,
                     point=None):
    dev = _cuda(sharedOut, maskedX, key, seed, point)
    es, N = maskedX.element_size(), maskedX.numel()
    sharedOut.resize_(out_shape)
    st = _Stream(dev)
    f = _lib.fn(op)
    if point is None:
        rc = f(_ptr(sharedOut), _nbytes(sharedOut), _ptr(maskedX), _nbytes(maskedX), _ptr(key), _nbytes(key),
               _ptr(seed), _nbytes(seed), partyId, bitWidthIn, bitWidthOut, groupSize, es, N, None, 0, st.ptr)
    else:
        rc = f(_ptr(sharedOut), _nbytes(sharedOut), _ptr(maskedX), _nbytes(maskedX), _ptr(key), _nbytes(key),
               _ptr(seed), _nbytes(seed), partyId, _ptr(point), _nbytes(point), bitWidthIn, bitWidthOut, groupSize,
               es, N, None, 0, st.ptr)
    _check(op, rc)
    return sharedOut


def dpf_eval(sharedOut, maskedX, key, seed, partyId, bitWidthIn, bitWidthOut, groupSize):
    return _dpf_eval_common("FastFss_cuda_dpfEval", sharedOut, list(maskedX.shape) + [groupSize], maskedX, key, seed,
                            partyId, bitWidthIn, bitWidthOut, groupSize)


def dpf_eval_all(sharedOut, maskedX, key, seed, partyId, bitWidthIn, bitWidthOut, groupSize):
    shape = list(maskedX.shape) + [1 << bitWidthIn, groupSize]
    return _dpf_eval_common("FastFss_cuda_dpfEvalAll", sharedOut, shape, maskedX, key, seed, partyId, bitWidthIn,
                            bitWidthOut, groupSize)


def dpf_multi_eval(sharedOut, maskedX, key, seed, partyId, point, bitWidthIn, bitWidthOut, groupSize):
    shape = list(maskedX.shape) + [point.numel(), groupSize]
    return _dpf_eval_common("FastFss_cuda_dpfEvalMulti", sharedOut, shape, maskedX, key, seed, partyId, bitWidthIn,
                            bitWidthOut, groupSize, point=point)


# ------------------------------------------------------------------------------------
# Grotto (bind_grotto.cpp)
# ------------------------------------------------------------------------------------

def grotto_get_key_data_size(bitWidthIn, elementSize, elementNum) -> int:
    return _size_query("FastFss_grottoGetKeyDataSize", bitWidthIn, elementSize, elementNum)


def grotto_key_gen(keyOut, alpha, seed0, seed1, bitWidthIn):
    dev = _cuda(keyOut, alpha, seed0, seed1)
    es, N = alpha.element_size(), alpha.numel()
    keyOut.resize_(grotto_get_key_data_size(bitWidthIn, es, N))
    st = _Stream(dev)
    _check("FastFss_cuda_grottoKeyGen", _lib.fn("FastFss_cuda_grottoKeyGen")(
        _ptr(keyOut), _nbytes(keyOut), _ptr(alpha), _nbytes(alpha), _ptr(seed0), _nbytes(seed0), _ptr(seed1),
        _nbytes(seed1), bitWidthIn, es, N, st.ptr))
    return keyOut


def grotto_eq_eval(sharedOut, maskedX, key, seed, partyId, bitWidthIn):
    dev = _cuda(sharedOut, maskedX, key, seed)
    es, N = maskedX.element_size(), maskedX.numel()
    sharedOut.resize_(maskedX.shape)
    st = _Stream(dev)
    _check("FastFss_cuda_grottoEqEval", _lib.fn("FastFss_cuda_grottoEqEval")(
        _ptr(sharedOut), _nbytes(sharedOut), _ptr(maskedX), _nbytes(maskedX), _ptr(key), _nbytes(key), _ptr(seed),
        _nbytes(seed), partyId, bitWidthIn, es, N, None, 0, st.ptr))
    return sharedOut


def grotto_eval(sharedOut, maskedX, key, seed, equalBound, partyId, bitWidthIn):
    dev = _cuda(sharedOut, maskedX, key, seed)
    es, N = maskedX.element_size(), maskedX.numel()
    sharedOut.resize_(maskedX.shape)
    st = _Stream(dev)
    _check("FastFss_cuda_grottoEval", _lib.fn("FastFss_cuda_grottoEval")(
        _ptr(sharedOut), _nbytes(sharedOut), _ptr(maskedX), _nbytes(maskedX), _ptr(key), _nbytes(key), _ptr(seed),
        _nbytes(seed), bool(equalBound), partyId, bitWidthIn, es, N, None, 0, st.ptr))
    return sharedOut


def grotto_mic_eval(sharedOut, maskedX, key, seed, partyId, leftBoundary, rightBoundary, bitWidthIn):
    dev = _cuda(sharedOut, maskedX, key, seed, leftBoundary, rightBoundary)
    es, N = maskedX.element_size(), maskedX.numel()
    sharedOut.resize_(list(maskedX.shape) + [leftBoundary.numel()])
    st = _Stream(dev)
    _check("FastFss_cuda_grottoMICEval", _lib.fn("FastFss_cuda_grottoMICEval")(
        _ptr(sharedOut), _nbytes(sharedOut), _ptr(maskedX), _nbytes(maskedX), _ptr(key), _nbytes(key), _ptr(seed),
        _nbytes(seed), partyId, _ptr(leftBoundary), _nbytes(leftBoundary), _ptr(rightBoundary),
        _nbytes(rightBoundary), bitWidthIn, es, N, None, 0, st.ptr))
    return sharedOut


def grotto_interval_lut_eval(sharedOutE, sharedOutT, maskedX, key, seed, partyId, leftBoundary, rightBoundary,
                             lookUpTable, bitWidthIn, bitWidthOut):
    dev = _cuda(sharedOutE, sharedOutT, maskedX, key, seed, leftBoundary, rightBoundary, lookUpTable)
    es, N = maskedX.element_size(), maskedX.numel()
    m = leftBoundary.numel()
    lut_num = lookUpTable.numel() // m if m else 0
    sharedOutE.resize_(maskedX.shape)
    sharedOutT.resize_(list(maskedX.shape) + [lut_num])
    st = _Stream(dev)
    _check("FastFss_cuda_grottoIntervalLutEval", _lib.fn("FastFss_cuda_grottoIntervalLutEval")(
        _ptr(sharedOutE), _nbytes(sharedOutE), _ptr(sharedOutT), _nbytes(sharedOutT), _ptr(maskedX),
        _nbytes(maskedX), _ptr(key), _nbytes(key), _ptr(seed), _nbytes(seed), partyId, _ptr(leftBoundary),
        _nbytes(leftBoundary), _ptr(rightBoundary), _nbytes(rightBoundary), _ptr(lookUpTable), _nbytes(lookUpTable),
        bitWidthIn, bitWidthOut, es, N, None, 0, st.ptr))
    return sharedOutE, sharedOutT


def _grotto_all(op, outBits, key, seed, partyId, bitWidthIn, elementSize, elementNum):
    dev = _cuda(outBits, key, seed)
    outBits.resize_(elementNum * (1 << bitWidthIn) // 8)
    st = _Stream(dev)
    _check(op, _lib.fn(op)(_ptr(outBits), _nbytes(outBits), _ptr(key), _nbytes(key), _ptr(seed), _nbytes(seed),
                           partyId, bitWidthIn, elementSize, elementNum, st.ptr))
    return outBits


def grotto_eq_eval_all(outBits, key, seed, partyId, bitWidthIn, elementSize, elementNum):
    """Full-domain Grotto equality shares: bit x of row i is grottoEqEval(key_i, x) (this
    library's extension, include/FastFss/b200/grotto_all.h)."""
    return _grotto_all("FastFss_cuda_grottoEqEvalAll", outBits, key, seed, partyId, bitWidthIn, elementSize,
                       elementNum)


def grotto_le_eval_all(outBits, key, seed, partyId, bitWidthIn, elementSize, elementNum):
    """Full-domain prefix-parity shares: bit x of row i is grottoEval(key_i, x, equalBound=true)."""
    return _grotto_all("FastFss_cuda_grottoLeEvalAll", outBits, key, seed, partyId, bitWidthIn, elementSize,
                       elementNum)


def grotto_interval_lut_eval_from_rows(sharedOutE, sharedOutT, maskedX, leRows, partyId, leftBoundary,
                                       rightBoundary, lookUpTable, bitWidthIn):
    """grotto_interval_lut_eval computed from full-domain comparison rows (grotto_le_eval_all
    output for the same keys/seeds/party): same shares, no tree walks."""
    dev = _cuda(sharedOutE, sharedOutT, maskedX, leRows, leftBoundary, rightBoundary, lookUpTable)
    es, N = maskedX.element_size(), maskedX.numel()
    m = leftBoundary.numel()
    lut_num = lookUpTable.numel() // m if m else 0
    sharedOutE.resize_(maskedX.shape)
    sharedOutT.resize_(list(maskedX.shape) + [lut_num])
    st = _Stream(dev)
    _check("FastFss_cuda_grottoIntervalLutEvalFromRows", _lib.fn("FastFss_cuda_grottoIntervalLutEvalFromRows")(
        _ptr(sharedOutE), _nbytes(sharedOutE), _ptr(sharedOutT), _nbytes(sharedOutT), _ptr(maskedX), _nbytes(maskedX),
        _ptr(leRows), _nbytes(leRows), partyId, _ptr(leftBoundary), _nbytes(leftBoundary), _ptr(rightBoundary),
        _nbytes(rightBoundary), _ptr(lookUpTable), _nbytes(lookUpTable), bitWidthIn, es, N, st.ptr))
    return sharedOutE, sharedOutT


# ------------------------------------------------------------------------------------
# DCF MIC (bind_dcf_mic.cpp)
# ------------------------------------------------------------------------------------

def dcf_mic_get_key_data_size(bitWidthIn, bitWidthOut, elementSize, elementNum) -> int:
    return _size_query("FastFss_dcfMICGetKeyDataSize", bitWidthIn, bitWidthOut, elementSize, elementNum)


def dcf_mic_key_gen(keyOut, zOut, alpha, seed0, seed1, leftBoundary, rightBoundary, bitWidthIn, bitWidthOut):
    dev = _cuda(keyOut, zOut, alpha, seed0, seed1, leftBoundary, rightBoundary)
    es, N = alpha.element_size(), alpha.numel()
    keyOut.resize_(dcf_mic_get_key_data_size(bitWidthIn, bitWidthOut, es, N))
    zOut.resize_(list(alpha.shape) + [leftBoundary.numel()])
    st = _Stream(dev)
    _check("FastFss_cuda_dcfMICKeyGen", _lib.fn("FastFss_cuda_dcfMICKeyGen")(
        _ptr(keyOut), _nbytes(keyOut), _ptr(zOut), _nbytes(zOut), _ptr(alpha), _nbytes(alpha), _ptr(seed0),
        _nbytes(seed0), _ptr(seed1), _nbytes(seed1), _ptr(leftBoundary), _nbytes(leftBoundary), _ptr(rightBoundary),
        _nbytes(rightBoundary), bitWidthIn, bitWidthOut, es, N, st.ptr))
    return keyOut, zOut


def dcf_mic_eval(sharedOut, maskedX, key, sharedZ, seed, partyId, leftBoundary, rightBoundary, bitWidthIn,
                 bitWidthOut):
    dev = _cuda(sharedOut, maskedX, key, sharedZ, seed, leftBoundary, rightBoundary)
    es, N = maskedX.element_size(), maskedX.numel()
    sharedOut.resize_(list(maskedX.shape) + [leftBoundary.numel()])
    st = _Stream(dev)
    _check("FastFss_cuda_dcfMICEval", _lib.fn("FastFss_cuda_dcfMICEval")(
        _ptr(sharedOut), _nbytes(sharedOut), _ptr(maskedX), _nbytes(maskedX), _ptr(key), _nbytes(key), _ptr(sharedZ),
        _nbytes(sharedZ), _ptr(seed), _nbytes(seed), partyId, _ptr(leftBoundary), _nbytes(leftBoundary),
        _ptr(rightBoundary), _nbytes(rightBoundary), bitWidthIn, bitWidthOut, es, N, None, 0, st.ptr))
    return sharedOut


# ------------------------------------------------------------------------------------
# spline (bind_spline.cpp)
# ------------------------------------------------------------------------------------

def spline_get_key_data_size(degree, intervalNum, bitWidthIn, bitWidthOut, elementSize, elementNum) -> int:
    return _size_query("FastFss_dcfSplineGetKeyDataSize", degree, intervalNum, bitWidthIn, bitWidthOut, elementSize,
                       elementNum)


def spline_get_cache_data_size(degree, intervalNum, bitWidthIn, bitWidthOut, elementSize, elementNum) -> int:
    return _size_query("FastFss_dcfSplineGetCacheDataSize", degree, intervalNum, bitWidthIn, bitWidthOut,
                       elementSize, elementNum)


def spline_key_gen(keyOut, eOut, betaOut, alpha, seed0, seed1, coefficients, degree, leftEndpoints, rightEndpoints,
                   intervalNum, bitWidthIn, bitWidthOut):
    dev = _cuda(keyOut, eOut, betaOut, alpha, seed0, seed1, coefficients, leftEndpoints, rightEndpoints)
    es, N = alpha.element_size(), alpha.numel()
    g = intervalNum * (degree + 1)
    keyOut.resize_(spline_get_key_data_size(degree, intervalNum, bitWidthIn, bitWidthOut, es, N))
    eOut.resize_(list(alpha.shape) + [g])
    betaOut.resize_(list(alpha.shape) + [g])
    st = _Stream(dev)
    _check("FastFss_cuda_dcfSplineKeyGen", _lib.fn("FastFss_cuda_dcfSplineKeyGen")(
        _ptr(keyOut), _nbytes(keyOut), _ptr(eOut), _nbytes(eOut), _ptr(betaOut), _nbytes(betaOut), _ptr(alpha),
        _nbytes(alpha), _ptr(seed0), _nbytes(seed0), _ptr(seed1), _nbytes(seed1), _ptr(coefficients),
        _nbytes(coefficients), degree, _ptr(leftEndpoints), _nbytes(leftEndpoints), _ptr(rightEndpoints),
        _nbytes(rightEndpoints), intervalNum, bitWidthIn, bitWidthOut, es, N, st.ptr))
    return keyOut, eOut, betaOut


def spline_eval(sharedOut, maskedX, key, sharedE, sharedBeta, seed, partyId, leftEndpoints, rightEndpoints,
                intervalNum, degree, bitWidthIn, bitWidthOut, cache=None):
    """The reference C ABI requires a per-element cache for spline evaluation
    (src/kernel/spline.h:202-205); this kernel never reads or writes it, so unless the caller
    passes one, a buffer of the required size is taken from torch's caching allocator."""
    dev = _cuda(sharedOut, maskedX, key, sharedE, sharedBeta, seed, leftEndpoints, rightEndpoints, cache)
    es, N = maskedX.element_size(), maskedX.numel()
    sharedOut.resize_(maskedX.shape)
    if cache is None:
        need = spline_get_cache_data_size(degree, intervalNum, bitWidthIn, bitWidthOut, es, N)
        cache = torch.empty(need, dtype=torch.uint8, device=dev)
    st = _Stream(dev)
    _check("FastFss_cuda_dcfSplineEval", _lib.fn("FastFss_cuda_dcfSplineEval")(
        _ptr(sharedOut), _nbytes(sharedOut), _ptr(maskedX), _nbytes(maskedX), _ptr(key), _nbytes(key), _ptr(sharedE),
        _nbytes(sharedE), _ptr(sharedBeta), _nbytes(sharedBeta), _ptr(seed), _nbytes(seed), partyId,
        _ptr(leftEndpoints), _nbytes(leftEndpoints), _ptr(rightEndpoints), _nbytes(rightEndpoints), intervalNum,
        degree, bitWidthIn, bitWidthOut, es, N, _ptr(cache), _nbytes(cache), st.ptr))
    return sharedOut


# ------------------------------------------------------------------------------------
# OTTT (bind_ottt.cpp)
# ------------------------------------------------------------------------------------

def ottt_get_key_data_size(bitWidthIn, elementNum) -> int:
    return _size_query("FastFss_otttGetKeyDataSize", bitWidthIn, elementNum)


def ottt_key_gen(keyInOut, alpha, bitWidthIn):
    dev = _cuda(keyInOut, alpha)
    es, N = alpha.element_size(), alpha.numel()
    st = _Stream(dev)
    _check("FastFss_cuda_otttKeyGen", _lib.fn("FastFss_cuda_otttKeyGen")(
        _ptr(keyInOut), _nbytes(keyInOut), _ptr(alpha), _nbytes(alpha), bitWidthIn, es, N, st.ptr))
    return keyInOut


def ottt_lut_eval(sharedOutE, sharedOutT, maskedX, key, partyId, lookUpTable, bitWidthIn, bitWidthOut):
    dev = _cuda(sharedOutE, sharedOutT, maskedX, key, lookUpTable)
    es, N = maskedX.element_size(), maskedX.numel()
    lut_num = lookUpTable.numel() // (1 << bitWidthIn)
    sharedOutE.resize_(maskedX.shape)
    sharedOutT.resize_(list(maskedX.shape) + [lut_num])
    st = _Stream(dev)
    _check("FastFss_cuda_otttLutEval", _lib.fn("FastFss_cuda_otttLutEval")(
        _ptr(sharedOutE), _nbytes(sharedOutE), _ptr(sharedOutT), _nbytes(sharedOutT), _ptr(maskedX), _nbytes(maskedX),
        _ptr(key), _nbytes(key), partyId, _ptr(lookUpTable), _nbytes(lookUpTable), bitWidthIn, es, N, st.ptr))
    return sharedOutE, sharedOutT


# ------------------------------------------------------------------------------------
# config (bind_config.cpp) and PRNG (pyFastPrng.cpp)
# ------------------------------------------------------------------------------------

def set_grid_dim(dim: int) -> None:
    _lib.fn("FastFss_cuda_setGridDim")(dim)


def get_grid_dim() -> int:
    return _lib.fn("FastFss_cuda_getGridDim")()


def set_fine_grain_parallel_grid_dim_threshold(dim: int) -> None:
    _lib.fn("FastFss_cuda_setFineGrainParallelGridDimThreshold")(dim)


def get_fine_grain_parallel_grid_dim_threshold() -> int:
    return _lib.fn("FastFss_cuda_getFineGrainParallelGridDimThreshold")()


class Prng:
    """AES-128-CTR generator on the GPU (FastFss_cuda_prng*), with the method set of the
    reference binding's ``pyFastFss.Prng`` (lib/torch_extension/pyFastFss/csrc/bind_prng.cpp:8-17,
    pyFastPrng.cpp): ``device()``, ``set_current_seed(seed128bit, counter128bit)``,
    ``get_current_seed()``, ``to_(device)``, ``rand_(out, bitWidth)``. CUDA devices only."""

    def __init__(self, device: torch.device | str = "cuda"):
        self._device = torch.device(device)
        if self._device.type != "cuda":
            raise ValueError("device not supported: FastFss-B200 runs on CUDA tensors only")
        self._h = self._init(self._device)

    @staticmethod
    def _init(device: torch.device):
        with torch.cuda.device(device):
            h = _lib.fn("FastFss_cuda_prngInit")()
        if not h:
            raise RuntimeError("FastFss_cuda_prngInit failed")
        return h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _lib.fn("FastFss_cuda_prngRelease")(h)
            self._h = None

    def device(self) -> torch.device:
        return self._device

    def set_current_seed(self, seed128bit: bytes, counter128bit: bytes) -> None:
        if len(seed128bit) != 16 or len(counter128bit) != 16:
            raise RuntimeError("seed128bit and counter128bit must be 16 bytes")
        _check("FastFss_cuda_prngSetCurrentSeed",
               _lib.fn("FastFss_cuda_prngSetCurrentSeed")(self._h, bytes(seed128bit), bytes(counter128bit)))

    def get_current_seed(self) -> tuple[bytes, bytes]:
        s, c = ctypes.create_string_buffer(16), ctypes.create_string_buffer(16)
        _check("FastFss_cuda_prngGetCurrentSeed", _lib.fn("FastFss_cuda_prngGetCurrentSeed")(self._h, s, c))
        return s.raw, c.raw

    def to_(self, device: torch.device | str) -> "Prng":
        """Moves the generator (seed and counter) to another CUDA device."""
        device = torch.device(device)
        if device.type != "cuda":
            raise ValueError("device not supported: FastFss-B200 runs on CUDA tensors only")
        seed, counter = self.get_current_seed()
        h = self._init(device)
        with torch.cuda.device(device):
            rc = _lib.fn("FastFss_cuda_prngSetCurrentSeed")(h, seed, counter)
        if rc != 0:
            _lib.fn("FastFss_cuda_prngRelease")(h)
            raise RuntimeError("FastFss_prngSetCurrentSeed failed")
        _lib.fn("FastFss_cuda_prngRelease")(self._h)
        self._h, self._device = h, device
        return self

    def rand_(self, out: torch.Tensor, bitWidth: int) -> torch.Tensor:
        """Fills `out` (values reduced to bitWidth bits) from the stream and returns it."""
        if not out.is_contiguous():
            raise ValueError("assert fail: out.is_contiguous()")
        if out.device.type != self._device.type:
            raise ValueError("assert fail: device_.type() == out.device().type()")
        if bitWidth > out.element_size() * 8:
            raise ValueError("assert fail: bitWidth <= elementSize * 8")
        st = _Stream(out.device)
        _check("FastFss_cuda_prngGen", _lib.fn("FastFss_cuda_prngGen")(
            self._h, _ptr(out), bitWidth, out.element_size(), out.numel(), st.ptr))
        return out
