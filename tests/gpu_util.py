"""Moves numpy ring arrays to CUDA tensors and back (bytes preserved; torch holds them in
the signed dtype of the same width, as pyFastFss callers do)."""

import numpy as np
import torch

SIGNED = {1: np.int8, 2: np.int16, 4: np.int32, 8: np.int64}
UNSIGNED = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}


def dev(a: np.ndarray) -> torch.Tensor:
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint8 and a.ndim == 1 and getattr(a, "_keep_u8", True):
        return torch.from_numpy(a.copy()).cuda()
    return torch.from_numpy(a.view(SIGNED[a.dtype.itemsize]).copy()).cuda()


def dev_bytes(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).cuda()


def dev_ring(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a).view(SIGNED[a.dtype.itemsize]).copy()).cuda()


def host(t: torch.Tensor, es: int | None = None) -> np.ndarray:
    a = t.detach().cpu().contiguous().numpy().reshape(-1)
    if es is None:
        es = a.dtype.itemsize
    return a.view(UNSIGNED[es])


def empty_ring(es: int) -> torch.Tensor:
    return torch.empty(0, dtype={1: torch.int8, 2: torch.int16, 4: torch.int32, 8: torch.int64}[es], device="cuda")


def empty_bytes() -> torch.Tensor:
    return torch.empty(0, dtype=torch.uint8, device="cuda")
