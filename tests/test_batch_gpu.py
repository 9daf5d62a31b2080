"""qcuInvertBatch: independent systems of uneven lattice, colour count, RHS count and
kappa solved together in one CUDA graph.

Each system's solution must equal what qcuInvert gives for that system alone (the same
kernels on the same data with deterministic reductions, so the iterates agree to
rounding), and its FP64 true residual ||b - M x|| / ||b||, recomputed by the oracle, must
meet the tolerance rule of the solver."""
import ctypes

import numpy as np
import pytest

import qcu_mrhs_b200 as q
from qcu_mrhs_b200 import fields as F
from tests.helpers import empty_dev, from_dev, rel_err, to_dev

pytestmark = pytest.mark.gpu

# lattice, n_color, m_rhs, kappa, seed
SYSTEMS = [
    ((4, 4, 4, 4), 3, 2, 0.10, 21),
    ((4, 4, 4, 8), 3, 3, 0.12, 22),
    ((6, 4, 4, 4), 2, 1, 0.11, 23),
    ((8, 8, 8, 8), 3, 4, 0.10, 24),
    ((4, 2, 2, 4), 4, 5, 0.115, 25),
    ((8, 8, 4, 8), 3, 12, 0.12, 26),   # the two-RHS packed kernel in the mixed solves
]
TOL = 1e-10


def _options(solver, **kw):
    o = q.default_options()
    o.solver = solver
    o.t_boundary = -1.0
    o.stop_true_residual = 1
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _fields(L, nc, m, seed):
    gauge = F.gauge_field(L, nc, seed, kind="smooth", eps=0.3)
    b = F.gaussian_fermions(L, nc, m, seed + 100)
    return gauge, b


def _single(L, nc, m, kappa, gauge, b, opts, max_iter):
    """The same system through the qcu.h path."""
    grid = q.QcuGrid((ctypes.c_int * 4)(1, 1, 1, 1))
    param = q.QcuParam((ctypes.c_int * 4)(*L))
    lib = q.lib()
    lib.initGridSize(ctypes.byref(grid), ctypes.byref(param), nc, m, q.DOUBLE, q.DOUBLE)
    q.check()
    dg = to_dev(gauge)
    lib.loadQcuGauge(dg.data_ptr(), q.DOUBLE)
    lib.getDslash(0, 1.0 / (2 * kappa) - 4.0)
    q.check(lib.qcuSetSolverOptions(ctypes.byref(opts)))
    vh = F.half_volume(L)
    ins = [to_dev(b[j]) for j in range(m)]
    outs = [empty_dev((2, vh, 4, nc)) for _ in range(m)]
    for j in range(m):
        lib.pushBackFermions(outs[j].data_ptr(), ins[j].data_ptr())
    lib.qcuInvert(max_iter, TOL)
    st = q.status()
    stats = q.solve_stats()
    lib.finalizeQcu()
    return np.stack([from_dev(o) for o in outs]), st, stats


def _batch(systems, opts, flags, max_iters=None):
    keep = []
    arr = (q.QcuBatchSystem * len(systems))()
    outs = []
    for i, (L, nc, m, kappa, gauge, b) in enumerate(systems):
        vh = F.half_volume(L)
        dg = to_dev(gauge)
        ins = [to_dev(b[j]) for j in range(m)]
        xs = [empty_dev((2, vh, 4, nc)) for _ in range(m)]
        bp = q.ptr_array([t.data_ptr() for t in ins])
        xp = q.ptr_array([t.data_ptr() for t in xs])
        keep += [dg, ins, xs, bp, xp]
        s = arr[i]
        s.lattice_size[:] = list(L)
        s.n_color, s.m_rhs, s.kappa, s.tol = nc, m, kappa, TOL
        s.max_iteration = 2000 if max_iters is None else max_iters[i]
        s.gauge = dg.data_ptr()
        s.b = ctypes.cast(bp, ctypes.POINTER(ctypes.c_void_p))
        s.x = ctypes.cast(xp, ctypes.POINTER(ctypes.c_void_p))
        outs.append(xs)
    rc = q.lib().qcuInvertBatch(arr, len(systems), ctypes.byref(opts), flags)
    xs = [np.stack([from_dev(t) for t in o]) for o in outs]
    return rc, arr, xs


def _true_rel(oracle_lib, x, gauge, b, L, kappa):
    m = b.shape[0]
    res = oracle_lib.mat(x, gauge, L, kappa, t_sign=-1.0) - b
    return np.linalg.norm(res.reshape(m, -1), axis=1) / np.linalg.norm(b.reshape(m, -1), axis=1)


@pytest.mark.parametrize("flags", [q.BATCH_DEVICE_LOOP, q.BATCH_HOST_LOOP], ids=["device_loop", "host_loop"])
@pytest.mark.parametrize("solver", [q.SOLVER_FUSED, q.SOLVER_MIXED], ids=["fp64", "mixed_bf16"])
def test_batch_matches_single_solves(oracle_lib, solver, flags):
    systems = []
    for L, nc, m, kappa, seed in SYSTEMS:
        gauge, b = _fields(L, nc, m, seed)
        systems.append((L, nc, m, kappa, gauge, b))
    opts = _options(solver)
    rc, arr, xs = _batch(systems, opts, flags)
    assert rc == q.SUCCESS, q.last_error()
    for i, (L, nc, m, kappa, gauge, b) in enumerate(systems):
        s = arr[i]
        assert s.status == q.SUCCESS
        tr = _true_rel(oracle_lib, xs[i], gauge, b, L, kappa)
        assert np.all(tr <= 2 * TOL), (i, tr)
        assert s.true_residual_max == pytest.approx(tr.max(), rel=1e-2, abs=1e-14)
        assert s.latency_seconds > 0
        x1, st1, stats1 = _single(L, nc, m, kappa, gauge, b, opts, 2000)
        assert st1 == q.SUCCESS
        assert s.iterations == stats1.iterations
        assert rel_err(xs[i], x1) <= 1e-12


def test_batch_reports_unconverged_system(oracle_lib):
    systems = []
    for L, nc, m, kappa, seed in SYSTEMS[:3]:
        gauge, b = _fields(L, nc, m, seed)
        systems.append((L, nc, m, kappa, gauge, b))
    rc, arr, xs = _batch(systems, _options(q.SOLVER_FUSED, check_interval=4), q.BATCH_DEVICE_LOOP,
                         max_iters=[2000, 3, 2000])
    assert rc == q.ERR_NOT_CONVERGED
    assert arr[0].status == q.SUCCESS and arr[2].status == q.SUCCESS
    assert arr[1].status == q.ERR_NOT_CONVERGED
    assert arr[1].iterations == 3
    for i in (0, 2):
        L, nc, m, kappa, gauge, b = systems[i]
        assert np.all(_true_rel(oracle_lib, xs[i], gauge, b, L, kappa) <= 2 * TOL)


def test_batch_autotunes_each_shape():
    lib = q.lib()
    systems = []
    for L, nc, m, kappa, seed in SYSTEMS[:2]:
        gauge, b = _fields(L, nc, m, seed)
        systems.append((L, nc, m, kappa, gauge, b))
    rc, arr, xs = _batch(systems, _options(q.SOLVER_MIXED), q.BATCH_DEVICE_LOOP)
    assert rc == q.SUCCESS, q.last_error()
    for L, nc, m, kappa, seed in SYSTEMS[:2]:
        assert lib.qcuGetTunedHop(nc, m, q.DOUBLE) > 0
        assert lib.qcuGetTunedHop(nc, m, q.BF16) > 0


def test_batch_reuses_kept_contexts(oracle_lib):
    """Two calls with QCU_BATCH_KEEP_CONTEXTS give the same solutions; the second reuses
    the first call's contexts; qcuBatchRelease frees them."""
    systems = []
    for L, nc, m, kappa, seed in SYSTEMS[:3]:
        gauge, b = _fields(L, nc, m, seed)
        systems.append((L, nc, m, kappa, gauge, b))
    opts = _options(q.SOLVER_MIXED)
    flags = q.BATCH_DEVICE_LOOP | q.BATCH_KEEP_CONTEXTS
    rc1, arr1, xs1 = _batch(systems, opts, flags)
    rc2, arr2, xs2 = _batch(systems, opts, flags)
    assert rc1 == q.SUCCESS and rc2 == q.SUCCESS, q.last_error()
    for i in range(len(systems)):
        assert arr1[i].iterations == arr2[i].iterations
        assert rel_err(xs2[i], xs1[i]) <= 1e-14
    assert q.lib().qcuBatchRelease() == q.SUCCESS
