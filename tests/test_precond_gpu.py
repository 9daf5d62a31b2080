"""Learned preconditioner kernels on the GPU against the oracle restatement:
the network output P b, the training loss and its weight gradient (forward, adjoint and
weight-gradient kernels), Adam steps that lower the loss, and the right-preconditioned
BiCGStab through qcuInvert (QCU_SOLVER_PRECOND), including its fallback to the plain
solver.  FP32 kernels vs FP64 oracle: tolerances are stated per check."""
import ctypes

import numpy as np
import pytest

import qcu_mrhs_b200 as q
from qcu_mrhs_b200 import fields as F
from qcu_mrhs_b200.precond import LearnedPreconditioner, identity_weights, layer_shapes
from tests.helpers import empty_dev, from_dev, rel_err, to_dev

pytestmark = pytest.mark.gpu


def _weights(layers, ch, seed, scale=0.15):
    rng = np.random.default_rng(seed)
    ws = identity_weights(layers, ch)
    return [w + scale * (rng.standard_normal(w.shape) + 1j * rng.standard_normal(w.shape)) for w in ws]


def _field(L, nc, m, seed):
    rng = np.random.default_rng(seed)
    vh = F.half_volume(L)
    return rng.standard_normal((2, vh, 4, nc, m)) + 1j * rng.standard_normal((2, vh, 4, nc, m))


@pytest.mark.parametrize("L,nc,m,layers,ch", [((4, 4, 4, 8), 3, 4, 4, 4), ((4, 2, 4, 4), 2, 3, 3, 2),
                                             ((4, 4, 2, 4), 4, 2, 2, 3), ((8, 4, 4, 4), 3, 8, 4, 8)])
def test_apply_matches_oracle(oracle_lib, L, nc, m, layers, ch):
    g = F.gauge_field(L, nc, 11)
    ws = _weights(layers, ch, 12)
    b = _field(L, nc, m, 13)
    P = LearnedPreconditioner(L, nc, m, layers, ch, t_boundary=-1.0)
    P.set_weights(ws)
    P.set_gauge(to_dev(g))
    out = to_dev(np.zeros_like(b))
    P.apply(out, to_dev(b))
    q.lib().qcuDeviceSynchronize()
    ref = oracle_lib.precond_apply(b, [w.astype(np.complex64).astype(np.complex128) for w in ws], g, L, -1.0)
    assert rel_err(from_dev(out), ref) <= 2e-5
    # FP32 fields give the same result
    out32 = to_dev(np.zeros_like(b), q.SINGLE)
    P.apply(out32, to_dev(b, q.SINGLE), precision=q.SINGLE)
    q.lib().qcuDeviceSynchronize()
    assert rel_err(from_dev(out32), ref) <= 2e-5
    P.close()


@pytest.mark.parametrize("L,nc,m,layers,ch", [((4, 4, 4, 4), 3, 2, 4, 3), ((4, 2, 2, 4), 2, 4, 2, 2)])
def test_loss_and_gradient_match_oracle(oracle_lib, L, nc, m, layers, ch):
    kappa = 0.12
    g = F.gauge_field(L, nc, 21, kind="smooth", eps=0.3)
    ws = [w.astype(np.complex64).astype(np.complex128) for w in _weights(layers, ch, 22, 0.1)]
    b = _field(L, nc, m, 23)
    P = LearnedPreconditioner(L, nc, m, layers, ch, t_boundary=-1.0)
    P.set_weights(ws)
    P.set_gauge(to_dev(g))
    loss, grads = P.loss_grad(to_dev(b), kappa)
    ref_loss, ref_grads = oracle_lib.precond_loss_grad(b, ws, g, L, kappa, -1.0)
    assert loss == pytest.approx(ref_loss, rel=1e-5)
    for gg, rg in zip(grads, ref_grads):
        assert rel_err(gg, rg) <= 1e-4
    P.close()


def test_training_lowers_the_loss():
    L, nc, m, kappa = (8, 4, 4, 8), 3, 4, 0.12
    g = F.gauge_field(L, nc, 31, kind="smooth", eps=0.3)
    P = LearnedPreconditioner(L, nc, m, 4, 4, t_boundary=-1.0)
    P.set_weights(identity_weights(4, 4, noise=0.01, seed=1))
    P.set_gauge(to_dev(g))
    bs = [to_dev(_field(L, nc, m, 40 + i)) for i in range(4)]
    first = [P.loss_grad(b, kappa, want_grad=False)[0] for b in bs]
    for epoch in range(15):
        for b in bs:
            P.train_step(b, kappa, 3e-3)
    last = [P.loss_grad(b, kappa, want_grad=False)[0] for b in bs]
    assert np.mean(last) < 0.7 * np.mean(first), (first, last)
    P.close()


def _setup_context(L, nc, m, kappa, gauge):
    grid = q.QcuGrid((ctypes.c_int * 4)(1, 1, 1, 1))
    param = q.QcuParam((ctypes.c_int * 4)(*L))
    lib = q.lib()
    lib.initGridSize(ctypes.byref(grid), ctypes.byref(param), nc, m, q.DOUBLE, q.DOUBLE)
    q.check()
    dg = to_dev(gauge)
    lib.loadQcuGauge(dg.data_ptr(), q.DOUBLE)
    lib.getDslash(0, 1.0 / (2 * kappa) - 4.0)
    q.check()
    return dg


def _invert(L, nc, m, b, solver, tol=1e-10):
    lib = q.lib()
    o = q.default_options()
    o.solver = solver
    o.t_boundary = -1.0
    o.stop_true_residual = 1
    q.check(lib.qcuSetSolverOptions(ctypes.byref(o)))
    vh = F.half_volume(L)
    ins = [to_dev(b[j]) for j in range(m)]
    outs = [empty_dev((2, vh, 4, nc)) for _ in range(m)]
    for j in range(m):
        lib.pushBackFermions(outs[j].data_ptr(), ins[j].data_ptr())
    lib.qcuInvert(2000, tol)
    st = q.status()
    msg = q.last_error()
    stats = q.solve_stats()
    _invert.message = msg
    return np.stack([from_dev(t) for t in outs]), st, stats


@pytest.mark.parametrize("trained", [False, True], ids=["identity_net", "trained_net"])
def test_preconditioned_solve(oracle_lib, trained):
    L, nc, m, kappa = (8, 8, 8, 8), 3, 4, 0.12
    gauge = F.gauge_field(L, nc, 51, kind="smooth", eps=0.3)
    b = F.gaussian_fermions(L, nc, m, 52)
    dg = _setup_context(L, nc, m, kappa, gauge)
    P = LearnedPreconditioner(L, nc, m, 4, 4, t_boundary=-1.0)
    P.set_weights(identity_weights(4, 4, noise=0.01, seed=2))
    P.set_gauge(dg)
    if trained:
        for i in range(30):
            P.train_step(to_dev(_field(L, nc, m, 60 + i % 6)), kappa, 3e-3)
    try:
        P.attach()
        x, st, stats = _invert(L, nc, m, b, q.SOLVER_PRECOND)
        assert st == q.SUCCESS, q.last_error()
        assert stats.fallback == 0
        assert stats.precond_iterations == stats.iterations > 0
        res = oracle_lib.mat(x, gauge, L, kappa, t_sign=-1.0) - b
        tr = np.linalg.norm(res.reshape(m, -1), axis=1) / np.linalg.norm(b.reshape(m, -1), axis=1)
        assert np.all(tr <= 2e-10), tr
        x_plain, st_p, stats_p = _invert(L, nc, m, b, q.SOLVER_FUSED)
        assert st_p == q.SUCCESS
        assert rel_err(x, x_plain) <= 1e-8
    finally:
        q.lib().qcuSetPreconditioner(None)
        q.lib().finalizeQcu()
        P.close()


def test_preconditioned_solve_falls_back_to_plain(oracle_lib):
    """A network of zero weights (P = 0) breaks BiCGStab down at once; the plain FP64
    solver then solves the system and the statistics say so."""
    L, nc, m, kappa = (4, 4, 4, 8), 3, 2, 0.11
    gauge = F.gauge_field(L, nc, 71, kind="smooth", eps=0.3)
    b = F.gaussian_fermions(L, nc, m, 72)
    dg = _setup_context(L, nc, m, kappa, gauge)
    P = LearnedPreconditioner(L, nc, m, 2, 2, t_boundary=-1.0)
    P.set_weights([np.zeros(s, dtype=np.complex128) for s in layer_shapes(2, 2)])
    try:
        P.attach()
        x, st, stats = _invert(L, nc, m, b, q.SOLVER_PRECOND)
        assert st == q.SUCCESS, q.last_error()
        assert stats.fallback == 1
        res = oracle_lib.mat(x, gauge, L, kappa, t_sign=-1.0) - b
        tr = np.linalg.norm(res.reshape(m, -1), axis=1) / np.linalg.norm(b.reshape(m, -1), axis=1)
        assert np.all(tr <= 2e-10)
    finally:
        q.lib().qcuSetPreconditioner(None)
        q.lib().finalizeQcu()
        P.close()


def test_attach_rejects_mismatched_network():
    L, nc, m, kappa = (4, 4, 4, 4), 3, 2, 0.11
    gauge = F.gauge_field(L, nc, 81)
    _setup_context(L, nc, m, kappa, gauge)
    P = LearnedPreconditioner(L, nc, m + 1, 2, 2)
    try:
        assert q.lib().qcuSetPreconditioner(P.handle) == q.ERR_INVALID
        o = q.default_options()
        o.solver = q.SOLVER_PRECOND
        q.check(q.lib().qcuSetSolverOptions(ctypes.byref(o)))
        b = F.gaussian_fermions(L, nc, m, 82)
        x, st, stats = _invert(L, nc, m, b, q.SOLVER_PRECOND)
        assert st == q.ERR_STATE and "preconditioner" in _invert.message
    finally:
        q.lib().finalizeQcu()
        P.close()


def test_trained_network_cuts_iterations_on_held_out_fields(oracle_lib):
    """What the network gains over the same method without it.  Pairs (b, x = M^-1 b) come
    from the plain FP64 solver on three seeded training fields; the network trains on the b
    of the pairs (loss sum_j ||M P b_j - b_j||^2 / ||b_j||^2) and its output approaches the
    solver's x.  On two held-out fields, right-preconditioned BiCGStab with the trained P
    needs clearly fewer iterations than with P = 1, at the same FP64 true residual."""
    L, nc, m, kappa, layers, ch = (8, 8, 8, 8), 3, 4, 0.124, 4, 4
    gather = lambda per_rhs: np.moveaxis(per_rhs, 0, -1).copy()   # [m][2][Vh][4][N] -> [2][Vh][4][N][m]
    pairs = []
    try:
        for f in range(3):
            gauge = F.gauge_field(L, nc, 300 + f, kind="smooth", eps=0.3)
            dg = _setup_context(L, nc, m, kappa, gauge)
            for k in range(3):
                b = F.gaussian_fermions(L, nc, m, 400 + 10 * f + k)
                x, st, _ = _invert(L, nc, m, b, q.SOLVER_FUSED)
                assert st == q.SUCCESS, q.last_error()
                pairs.append((f, dg, gather(b), gather(x)))
            q.lib().finalizeQcu()
        P = LearnedPreconditioner(L, nc, m, layers, ch, t_boundary=-1.0)
        P.set_weights(identity_weights(layers, ch, noise=0.01, seed=3))

        def fit():   # ||P b - x|| / ||x|| over the pairs
            errs = []
            for _, dg, b, x in pairs:
                P.set_gauge(dg)
                y = to_dev(np.zeros_like(b))
                P.apply(y, to_dev(b))
                q.lib().qcuDeviceSynchronize()
                errs.append(rel_err(from_dev(y), x))
            return float(np.mean(errs))

        fit0 = fit()
        rng = np.random.default_rng(5)
        for epoch in range(12):
            lr = 3e-3 * (0.5 ** (epoch // 4))
            for i in rng.permutation(len(pairs)):
                _, dg, b, _ = pairs[i]
                P.set_gauge(dg)
                P.train_step(to_dev(b), kappa, lr)
        fit1 = fit()
        assert fit1 < 0.7 * fit0, (fit0, fit1)
        ident = LearnedPreconditioner(L, nc, m, layers, ch, t_boundary=-1.0)
        ident.set_weights(identity_weights(layers, ch))
        iters = {"identity": [], "learned": []}
        for f in range(2):
            gauge = F.gauge_field(L, nc, 900 + f, kind="smooth", eps=0.3)
            b = F.gaussian_fermions(L, nc, m, 950 + f)
            dg = _setup_context(L, nc, m, kappa, gauge)
            for name, net in (("identity", ident), ("learned", P)):
                net.set_gauge(dg)
                net.attach()
                x, st, stats = _invert(L, nc, m, b, q.SOLVER_PRECOND)
                assert st == q.SUCCESS, q.last_error()
                assert stats.fallback == 0
                res = oracle_lib.mat(x, gauge, L, kappa, t_sign=-1.0) - b
                tr = np.linalg.norm(res.reshape(m, -1), axis=1) / np.linalg.norm(b.reshape(m, -1), axis=1)
                assert np.all(tr <= 2e-10), tr
                iters[name].append(stats.iterations)
                q.lib().qcuSetPreconditioner(None)
            q.lib().finalizeQcu()
        print("fit", fit0, fit1, "iterations", iters)
        assert np.mean(iters["learned"]) <= 0.75 * np.mean(iters["identity"]), iters
        P.close()
        ident.close()
    finally:
        q.lib().qcuSetPreconditioner(None)
        q.lib().finalizeQcu()
