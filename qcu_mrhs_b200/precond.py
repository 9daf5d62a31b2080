"""Python handle of the learned gauge-covariant preconditioner (qcuPrecond* in
include/qcu_b200.h).  All compute runs in libqcu_b200.so; this class only packs weights
and passes device pointers.

Weights are a list with one complex array [cout][cin][9][4][4] per layer
(path 0 identity, 1 + 2 mu forward hop, 2 + 2 mu backward hop); fields are gathered
full-lattice multi-RHS spinors [2][Vh][4][N][m] as device tensors (FP32 or FP64,
complex stored as a trailing dimension of 2).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import SINGLE, DOUBLE, check, lattice, lib


def layer_shapes(layers: int, channels: int):
    shapes = []
    for l in range(layers):
        cin = 1 if l == 0 else channels
        cout = 1 if l == layers - 1 else channels
        shapes.append((cout, cin, 9, 4, 4))
    return shapes


def identity_weights(layers: int, channels: int, scale: float = 1.0, noise: float = 0.0, seed: int = 0):
    """Weights of P = scale * 1 (channel 0 passes the field through identity paths),
    plus optional small Gaussian noise on every weight."""
    rng = np.random.default_rng(seed)
    ws = []
    for l, shp in enumerate(layer_shapes(layers, channels)):
        w = np.zeros(shp, dtype=np.complex128)
        w[0, 0, 0] = np.eye(4) * (scale if l == 0 else 1.0)
        if noise:
            w += noise * (rng.standard_normal(shp) + 1j * rng.standard_normal(shp))
        ws.append(w)
    return ws


class LearnedPreconditioner:
    def __init__(self, L, n_color: int, m_rhs: int, layers: int = 4, channels: int = 8, t_boundary: float = 1.0):
        self.L, self.nc, self.m = tuple(L), n_color, m_rhs
        self.layers, self.channels = layers, channels
        h = ctypes.c_void_p()
        check(lib().qcuPrecondCreate(ctypes.byref(h), lattice(L), n_color, m_rhs, layers, channels, t_boundary))
        self.handle = h
        self.nw = int(lib().qcuPrecondNumWeights(h))

    def close(self):
        if self.handle:
            lib().qcuPrecondDestroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- weights ----
    def set_weights(self, ws):
        flat = np.concatenate([np.asarray(w, dtype=np.complex128).reshape(-1) for w in ws])
        assert flat.size == self.nw, (flat.size, self.nw)
        buf = np.ascontiguousarray(flat.astype(np.complex64)).view(np.float32)
        check(lib().qcuPrecondSetWeights(self.handle, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))

    def get_weights(self):
        buf = np.empty(2 * self.nw, dtype=np.float32)
        check(lib().qcuPrecondGetWeights(self.handle, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        flat = buf.view(np.complex64).astype(np.complex128)
        out, off = [], 0
        for shp in layer_shapes(self.layers, self.channels):
            n = int(np.prod(shp))
            out.append(flat[off:off + n].reshape(shp))
            off += n
        return out

    # ---- fields ----
    def set_gauge(self, gauge_dev, precision=DOUBLE):
        check(lib().qcuPrecondSetGauge(self.handle, gauge_dev.data_ptr(), precision))

    def apply(self, out_dev, in_dev, precision=DOUBLE, stream=None):
        check(lib().qcuPrecondApply(self.handle, out_dev.data_ptr(), in_dev.data_ptr(), precision, stream))

    def loss_grad(self, b_dev, kappa, precision=DOUBLE, want_grad=True):
        loss = ctypes.c_double()
        grad = np.empty(2 * self.nw, dtype=np.float64) if want_grad else None
        gp = grad.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if want_grad else None
        check(lib().qcuPrecondLossGrad(self.handle, b_dev.data_ptr(), precision, kappa, ctypes.byref(loss), gp))
        if not want_grad:
            return loss.value, None
        flat = grad[0::2] + 1j * grad[1::2]
        out, off = [], 0
        for shp in layer_shapes(self.layers, self.channels):
            n = int(np.prod(shp))
            out.append(flat[off:off + n].reshape(shp))
            off += n
        return loss.value, out

    def train_step(self, b_dev, kappa, lr, precision=DOUBLE):
        loss = ctypes.c_double()
        check(lib().qcuPrecondTrainStep(self.handle, b_dev.data_ptr(), precision, kappa, lr, ctypes.byref(loss)))
        return loss.value

    def attach(self):
        """Use this network for QCU_SOLVER_PRECOND solves of the current qcu.h context."""
        check(lib().qcuSetPreconditioner(self.handle))
