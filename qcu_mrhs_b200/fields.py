"""Seeded synthetic lattice fields: SU(N) links and complex Gaussian sources.

The reference has no field generator of its own (its gauge comes from a file
reader in an external submodule, src/qcu_interface.cu:364-411), so these are
written from the definitions of the ensembles the benchmark configurations name:

* Haar-random SU(N): QR of an N x N complex Gaussian matrix, columns rephased by
  the phases of R's diagonal (Mezzadri's recipe), then the determinant phase
  divided out so that det U = 1.
* smoothed links U = exp(i eps H), H a traceless Hermitian Gaussian matrix;
  computed by diagonalising H (U = V diag(exp(i eps lambda)) V^dagger).
* sources: unit complex Gaussian entries (E|z|^2 = 1).

Layouts follow the reference's even/odd convention (include/point/qcu_point.cuh:68-81):
gauge  [mu=4][parity=2][Vh][N][N] complex, fermion [parity=2][Vh][Ns=4][N] complex,
half-site index ((t*Lz + z)*Ly + y)*(Lx/2) + xh and full x = 2*xh + ((p+y+z+t) & 1).
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "half_volume",
    "haar_sun",
    "smoothed_sun",
    "gauge_field",
    "fold_t_boundary",
    "gaussian_fermions",
    "to_mrhs",
    "from_mrhs",
]


def half_volume(L) -> int:
    Lx, Ly, Lz, Lt = (int(v) for v in L)
    if Lx % 2:
        raise ValueError("Lx must be even for the even/odd layout")
    return Lx * Ly * Lz * Lt // 2


def _complex_gaussian(rng: np.random.Generator, shape, scale=1.0) -> np.ndarray:
    n = int(np.prod(shape))
    z = rng.standard_normal(size=2 * n)          # interleaved (re, im)
    z *= scale / np.sqrt(2.0)
    return z.view(np.complex128).reshape(tuple(shape))


def haar_sun(rng: np.random.Generator, count: int, n: int, chunk: int = 1 << 18) -> np.ndarray:
    """count Haar-random SU(n) matrices, shape (count, n, n) complex128."""
    out = np.empty((count, n, n), dtype=np.complex128)
    for s in range(0, count, chunk):
        e = min(count, s + chunk)
        z = _complex_gaussian(rng, (e - s, n, n))
        q, r = np.linalg.qr(z)
        d = np.diagonal(r, axis1=-2, axis2=-1)
        q = q * (d / np.abs(d))[:, None, :]
        det = np.linalg.det(q)
        q = q / (det ** (1.0 / n))[:, None, None]
        out[s:e] = q
    return out


def smoothed_sun(rng: np.random.Generator, count: int, n: int, eps: float,
                 chunk: int = 1 << 18) -> np.ndarray:
    """count matrices exp(i eps H), H traceless Hermitian Gaussian; shape (count, n, n)."""
    out = np.empty((count, n, n), dtype=np.complex128)
    eye = np.eye(n)
    for s in range(0, count, chunk):
        e = min(count, s + chunk)
        a = _complex_gaussian(rng, (e - s, n, n))
        h = 0.5 * (a + np.conj(np.swapaxes(a, -1, -2)))
        tr = np.trace(h, axis1=-2, axis2=-1).real / n
        h = h - tr[:, None, None] * eye
        lam, v = np.linalg.eigh(h)
        ph = np.exp(1j * eps * lam)
        out[s:e] = (v * ph[:, None, :]) @ np.conj(np.swapaxes(v, -1, -2))
    return out


def gauge_field(L, n: int, seed: int, kind: str = "haar", eps: float = 0.3) -> np.ndarray:
    """Even/odd gauge field [4][2][Vh][n][n] complex128 (links generated in storage order)."""
    vh = half_volume(L)
    rng = np.random.default_rng(seed)
    count = 4 * 2 * vh
    if kind == "haar":
        u = haar_sun(rng, count, n)
    elif kind == "smooth":
        u = smoothed_sun(rng, count, n, eps)
    elif kind == "unit":
        u = np.broadcast_to(np.eye(n, dtype=np.complex128), (count, n, n)).copy()
    else:
        raise ValueError(f"unknown gauge kind {kind!r}")
    return u.reshape(4, 2, vh, n, n)


def fold_t_boundary(gauge: np.ndarray, L, sign: float = -1.0) -> np.ndarray:
    """Return a copy with the t-links on the last time slice multiplied by `sign`.

    With sign = -1 the periodic hop on the folded field equals the antiperiodic-in-t
    hop on the original field.
    """
    Lx, Ly, Lz, Lt = (int(v) for v in L)
    g = gauge.copy()
    vh = half_volume(L)
    idx = np.arange(vh)
    t = idx // ((Lx // 2) * Ly * Lz)
    sel = t == Lt - 1
    g[3, :, sel] *= sign
    return g


def gaussian_fermions(L, n: int, m: int, seed: int, parities: int = 2) -> np.ndarray:
    """m per-RHS even/odd fermions [m][parities][Vh][4][n] complex128, unit Gaussian."""
    vh = half_volume(L)
    rng = np.random.default_rng(seed)
    return _complex_gaussian(rng, (m, parities, vh, 4, n))


def to_mrhs(per_rhs: np.ndarray) -> np.ndarray:
    """[m][Vh][4][n] -> gathered [Vh][4][n][m] (reference copy_color_spinor.cuh:27-37)."""
    return np.ascontiguousarray(np.moveaxis(per_rhs, 0, -1))


def from_mrhs(mrhs: np.ndarray) -> np.ndarray:
    """gathered [Vh][4][n][m] -> [m][Vh][4][n]."""
    return np.ascontiguousarray(np.moveaxis(mrhs, -1, 0))


# ---------------- device-side generators (same ensembles, torch RNG on the GPU) ----------------

def gauge_field_torch(L, n: int, seed: int, kind: str = "smooth", eps: float = 0.3, device="cuda"):
    """Even/odd gauge field [4][2][Vh][n][n] complex128 generated on `device`
    (torch Philox stream, so values differ from the numpy generator of the same seed)."""
    import torch
    vh = half_volume(L)
    count = 8 * vh
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    out = torch.empty((count, n, n), dtype=torch.complex128, device=device)
    chunk = 1 << 20
    eye = torch.eye(n, dtype=torch.complex128, device=device)
    for s in range(0, count, chunk):
        e = min(count, s + chunk)
        a = torch.randn((e - s, n, n, 2), dtype=torch.float64, device=device, generator=g) / np.sqrt(2.0)
        a = torch.view_as_complex(a)
        if kind == "smooth":
            h = 0.5 * (a + a.conj().transpose(-1, -2))
            tr = torch.diagonal(h, dim1=-2, dim2=-1).sum(-1).real / n
            h = h - tr[:, None, None] * eye
            lam, v = torch.linalg.eigh(h)
            ph = torch.exp(1j * eps * lam.to(torch.complex128))
            out[s:e] = (v * ph[:, None, :]) @ v.conj().transpose(-1, -2)
        elif kind == "haar":
            q, r = torch.linalg.qr(a)
            d = torch.diagonal(r, dim1=-2, dim2=-1)
            q = q * (d / d.abs())[:, None, :]
            det = torch.linalg.det(q)
            out[s:e] = q / (det ** (1.0 / n))[:, None, None]
        else:
            raise ValueError(f"unknown gauge kind {kind!r}")
    return out.reshape(4, 2, vh, n, n)


def gaussian_fermions_torch(L, n: int, m: int, seed: int, device="cuda"):
    """m per-RHS even/odd fermions [m][2][Vh][4][n] complex128, unit Gaussian, on `device`."""
    import torch
    vh = half_volume(L)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    z = torch.randn((m, 2, vh, 4, n, 2), dtype=torch.float64, device=device, generator=g)
    z /= np.sqrt(2.0)
    return torch.view_as_complex(z)
