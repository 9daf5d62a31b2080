"""The learned preconditioner's CPU restatement (oracle_ptc_*), checked from its
definition: the adjoint identity, finite-difference gradients of the training loss,
gauge covariance, and the identity network.  These pin the oracle that the GPU kernels
are compared with in test_precond_gpu.py."""
import numpy as np
import pytest

from qcu_mrhs_b200 import fields as F


def _rnd(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def identity_weights(layers, ch, scale=1.0):
    """P = scale * 1: channel 0 carries the field through identity paths."""
    ws = []
    for l in range(layers):
        cin = 1 if l == 0 else ch
        cout = 1 if l == layers - 1 else ch
        w = np.zeros((cout, cin, 9, 4, 4), dtype=np.complex128)
        w[0, 0, 0] = np.eye(4) * (scale if l == 0 else 1.0)
        ws.append(w)
    return ws


def test_layer_adjoint_identity(oracle_lib):
    O = oracle_lib
    L, nc, m = (4, 2, 4, 4), 3, 2
    vh = F.half_volume(L)
    rng = np.random.default_rng(1)
    g = F.gauge_field(L, nc, 5)
    a = _rnd(rng, 2, 2, vh, 4, nc, m)
    w = _rnd(rng, 3, 2, 9, 4, 4)
    b = _rnd(rng, 3, 2, vh, 4, nc, m)
    for t_sign in (1.0, -1.0):
        lhs = np.vdot(b, O.ptc_forward(a, w, g, L, t_sign))
        rhs = np.vdot(O.ptc_adjoint(b, w, g, L, t_sign), a)
        assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_loss_gradient_matches_finite_differences(oracle_lib):
    O = oracle_lib
    L, nc, m, kappa = (4, 4, 2, 4), 3, 2, 0.12
    vh = F.half_volume(L)
    rng = np.random.default_rng(2)
    g = F.gauge_field(L, nc, 6)
    ws = [0.1 * _rnd(rng, 2, 1, 9, 4, 4), 0.1 * _rnd(rng, 2, 2, 9, 4, 4), 0.1 * _rnd(rng, 1, 2, 9, 4, 4)]
    b = _rnd(rng, 2, vh, 4, nc, m)
    loss, grads = O.precond_loss_grad(b, ws, g, L, kappa, -1.0)
    h = 1e-6
    for li, idx in [(0, (1, 0, 3, 2, 1)), (1, (0, 1, 5, 0, 3)), (2, (0, 0, 0, 1, 1)), (1, (1, 1, 8, 3, 0))]:
        for part in (1.0, 1j):
            wp = [w.copy() for w in ws]
            wm = [w.copy() for w in ws]
            wp[li][idx] += h * part
            wm[li][idx] -= h * part
            fd = (O.precond_loss_grad(b, wp, g, L, kappa, -1.0)[0] - O.precond_loss_grad(b, wm, g, L, kappa, -1.0)[0]) / (2 * h)
            an = grads[li][idx].real if part == 1.0 else grads[li][idx].imag
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (li, idx, part, fd, an)


def test_network_is_gauge_covariant(oracle_lib):
    O = oracle_lib
    L, nc, m = (4, 4, 2, 6), 3, 2
    Lx, Ly, Lz, Lt = L
    vh = F.half_volume(L)
    rng = np.random.default_rng(3)
    gauge = F.gauge_field(L, nc, 7)
    om = F.haar_sun(np.random.default_rng(4), 2 * vh, nc).reshape(2, vh, nc, nc)

    def fwd(par, idx, mu):
        xh = idx % (Lx // 2); q = idx // (Lx // 2)
        yy = q % Ly; q //= Ly
        zz = q % Lz; tt = q // Lz
        c = [2 * xh + ((par + yy + zz + tt) & 1), yy, zz, tt]
        c[mu] = (c[mu] + 1) % L[mu]
        return ((c[3] * Lz + c[2]) * Ly + c[1]) * (Lx // 2) + c[0] // 2

    g2 = np.empty_like(gauge)
    idx = np.arange(vh)
    for mu in range(4):
        for par in range(2):
            g2[mu, par] = om[par] @ gauge[mu, par] @ np.conj(np.swapaxes(om[1 - par][fwd(par, idx, mu)], -1, -2))
    ws = [0.3 * _rnd(rng, 3, 1, 9, 4, 4), 0.3 * _rnd(rng, 3, 3, 9, 4, 4), 0.3 * _rnd(rng, 1, 3, 9, 4, 4)]
    b = _rnd(rng, 2, vh, 4, nc, m)
    rot = lambda v: np.einsum("pvab,pvsbm->pvsam", om, v)
    for t_sign in (1.0, -1.0):
        y = O.precond_apply(b, ws, gauge, L, t_sign)
        y2 = O.precond_apply(rot(b), ws, g2, L, t_sign)
        assert np.abs(y2 - rot(y)).max() <= 1e-11 * np.abs(y).max()


def test_identity_network(oracle_lib):
    O = oracle_lib
    L, nc, m = (4, 2, 2, 4), 2, 3
    vh = F.half_volume(L)
    rng = np.random.default_rng(5)
    g = F.gauge_field(L, nc, 8)
    b = _rnd(rng, 2, vh, 4, nc, m)
    assert np.allclose(O.precond_apply(b, identity_weights(4, 3, 0.7), g, L, -1.0), 0.7 * b, atol=1e-14)
