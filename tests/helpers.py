"""Test helpers: seeded fields, device buffers in each storage precision."""
from __future__ import annotations

import numpy as np

import qcu_mrhs_b200 as q

TORCH_REAL = None


def _torch():
    import torch
    return torch


def real_dtype(prec):
    torch = _torch()
    return {q.DOUBLE: torch.float64, q.SINGLE: torch.float32, q.HALF: torch.float16,
            q.BF16: torch.bfloat16}[prec]


def to_dev(arr: np.ndarray, prec=q.DOUBLE):
    """complex numpy array -> CUDA tensor [..., 2] of the storage type of `prec`."""
    torch = _torch()
    a = np.ascontiguousarray(arr, dtype=np.complex128)
    t = torch.from_numpy(a.view(np.float64).reshape(a.shape + (2,)).copy())
    return t.to(device="cuda", dtype=real_dtype(prec)).contiguous()


def from_dev(t) -> np.ndarray:
    a = t.detach().to(device="cpu", dtype=_torch().float64).numpy()
    return a[..., 0] + 1j * a[..., 1]


def empty_dev(shape, prec=q.DOUBLE):
    torch = _torch()
    return torch.empty(tuple(shape) + (2,), dtype=real_dtype(prec), device="cuda")


def zeros_dev(shape, prec=q.DOUBLE):
    torch = _torch()
    return torch.zeros(tuple(shape) + (2,), dtype=real_dtype(prec), device="cuda")


def rel_err(a, b) -> float:
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def sync():
    _torch().cuda.synchronize()
