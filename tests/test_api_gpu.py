"""The qcu.h flow on the GPU, used the way the reference's callers use it
(initGridSize -> loadQcuGauge -> getDslash -> pushBackFermions x m ->
start_dslash | mat_Qcu | qcuInvert -> finalizeQcu), checked against the oracle."""
import ctypes

import numpy as np
import pytest
import torch

import qcu_mrhs_b200 as q
from qcu_mrhs_b200 import fields as F
from tests.helpers import empty_dev, from_dev, rel_err, sync, to_dev

pytestmark = pytest.mark.gpu


def init(L, nc, m, in_prec=q.DOUBLE, dslash_prec=q.DOUBLE):
    grid = q.QcuGrid((ctypes.c_int * 4)(1, 1, 1, 1))
    param = q.QcuParam((ctypes.c_int * 4)(*L))
    q.lib().initGridSize(ctypes.byref(grid), ctypes.byref(param), nc, m, in_prec, dslash_prec)
    q.check()


@pytest.fixture(autouse=True)
def _finalize():
    yield
    q.lib().qcuSetHopKernel(q.HOP_AUTO)
    q.lib().finalizeQcu()


def _setup(L, nc, m, kappa, seed, in_prec=q.DOUBLE, dslash_prec=q.DOUBLE, kind="haar"):
    init(L, nc, m, in_prec, dslash_prec)
    gauge = F.gauge_field(L, nc, seed, kind=kind, eps=0.3)
    dg = to_dev(gauge, in_prec)
    q.lib().loadQcuGauge(dg.data_ptr(), in_prec)
    q.check()
    q.lib().getDslash(0, 1.0 / (2 * kappa) - 4.0)
    q.check()
    return gauge, dg


@pytest.mark.parametrize("dagger", [0, 1])
def test_start_dslash(oracle_lib, dagger):
    L, nc, m = (8, 8, 8, 8), 3, 4
    gauge, dg = _setup(L, nc, m, 0.1, 1)
    vh = F.half_volume(L)
    psi = F.gaussian_fermions(L, nc, m, 2, parities=1)[:, 0]
    ins = [to_dev(psi[j]) for j in range(m)]
    for parity in (0, 1):
        outs = [empty_dev((vh, 4, nc)) for _ in range(m)]
        for j in range(m):
            q.lib().pushBackFermions(outs[j].data_ptr(), ins[j].data_ptr())
        q.lib().start_dslash(parity, dagger)
        q.check()
        got = np.stack([from_dev(o) for o in outs])
        ref = F.from_mrhs(oracle_lib.hop(F.to_mrhs(psi), gauge, L, parity, bool(dagger)))
        assert rel_err(got, ref) <= 1e-13


@pytest.mark.parametrize("dagger", [0, 1])
def test_mat_qcu(oracle_lib, dagger):
    L, nc, m, kappa = (8, 4, 4, 8), 3, 3, 0.12
    gauge, dg = _setup(L, nc, m, kappa, 3)
    vh = F.half_volume(L)
    psi = F.gaussian_fermions(L, nc, m, 4)
    ins = [to_dev(psi[j]) for j in range(m)]
    outs = [empty_dev((2, vh, 4, nc)) for _ in range(m)]
    for j in range(m):
        q.lib().pushBackFermions(outs[j].data_ptr(), ins[j].data_ptr())
    q.lib().mat_Qcu(dagger)
    q.check()
    got = np.stack([from_dev(o) for o in outs])
    ref = oracle_lib.mat(psi, gauge, L, kappa, bool(dagger))
    assert rel_err(got, ref) <= 1e-13


def test_mat_qcu_half_precision_dslash(oracle_lib):
    L, nc, m, kappa = (8, 4, 4, 4), 3, 2, 0.11
    gauge, dg = _setup(L, nc, m, kappa, 5, dslash_prec=q.HALF)
    vh = F.half_volume(L)
    psi = F.gaussian_fermions(L, nc, m, 6)
    ins = [to_dev(psi[j]) for j in range(m)]
    outs = [empty_dev((2, vh, 4, nc)) for _ in range(m)]
    for j in range(m):
        q.lib().pushBackFermions(outs[j].data_ptr(), ins[j].data_ptr())
    q.lib().mat_Qcu(0)
    q.check()
    got = np.stack([from_dev(o) for o in outs])
    assert rel_err(got, oracle_lib.mat(psi, gauge, L, kappa)) <= 3e-3


def _round(arr, prec):
    """Round a complex array to a 16-bit storage format and back (torch on CPU)."""
    import torch
    dt = {q.HALF: torch.float16, q.BF16: torch.bfloat16}[prec]
    a = np.ascontiguousarray(arr, dtype=np.complex128)
    t = torch.from_numpy(a.view(np.float64).reshape(a.shape + (2,)).copy()).to(dt).to(torch.float64).numpy()
    return t[..., 0] + 1j * t[..., 1]


@pytest.mark.parametrize("prec", [q.HALF, q.BF16])
@pytest.mark.parametrize("t_boundary", [1.0, -1.0])
@pytest.mark.parametrize("m", [4, 12, 7])
def test_start_dslash_and_mat_low_precision_tables(oracle_lib, prec, t_boundary, m):
    """16-bit start_dslash and mat_Qcu on a context: with the automatic kernel choice the hop
    is the link-operand tensor-core kernel, which on a context reads the per-site neighbour
    table and hop-link array (t-boundary sign folded in) instead of recomputing them.  Both
    parities, dagger, both t boundaries, against the oracle on the same rounded inputs."""
    L, nc, kappa = (8, 4, 4, 6), 3, 0.11
    tol = {q.HALF: 2e-3, q.BF16: 1.5e-2}[prec]
    gauge, dg = _setup(L, nc, m, kappa, 21, dslash_prec=prec)
    o = q.default_options()
    o.t_boundary = t_boundary
    q.check(q.lib().qcuSetSolverOptions(ctypes.byref(o)))
    vh = F.half_volume(L)
    gr = _round(gauge, prec)
    psi = F.gaussian_fermions(L, nc, m, 22, parities=1)[:, 0]
    ins = [to_dev(psi[j]) for j in range(m)]
    for dagger in (0, 1):
        for parity in (0, 1):
            outs = [empty_dev((vh, 4, nc)) for _ in range(m)]
            for j in range(m):
                q.lib().pushBackFermions(outs[j].data_ptr(), ins[j].data_ptr())
            q.lib().start_dslash(parity, dagger)
            q.check()
            got = np.stack([from_dev(x) for x in outs])
            ref = F.from_mrhs(oracle_lib.hop(_round(F.to_mrhs(psi), prec), gr, L, parity, bool(dagger), t_boundary))
            assert rel_err(got, ref) <= tol
    full = F.gaussian_fermions(L, nc, m, 23)
    fins = [to_dev(full[j]) for j in range(m)]
    for dagger in (0, 1):
        outs = [empty_dev((2, vh, 4, nc)) for _ in range(m)]
        for j in range(m):
            q.lib().pushBackFermions(outs[j].data_ptr(), fins[j].data_ptr())
        q.lib().mat_Qcu(dagger)
        q.check()
        got = np.stack([from_dev(x) for x in outs])
        ref = oracle_lib.mat(full, gauge, L, kappa, bool(dagger), t_boundary)
        assert rel_err(got, ref) <= tol
    assert q.lib().qcuGetKernelError(1) == 0


@pytest.mark.parametrize("kind", [q.HOP_AUTO, q.HOP_MMA_LINK_DIRECT], ids=["auto", "mma_link_direct"])
@pytest.mark.parametrize("prec", [q.HALF, q.BF16, q.DOUBLE])
@pytest.mark.parametrize("m", [4, 8, 12, 16, 6])
def test_context_hop(oracle_lib, prec, m, kind):
    """qcuDslashMrhsContext: the context's own hop (gauge copy, t boundary, and for FP16/BF16
    the per-site tables; m = 4, 8, 12, 16 run the shared-memory staged tensor-core kernel) on
    caller gathered fields, both parities and dagger, against the oracle on the same
    rounded inputs; the same call twice gives the same bits (the tables are reused)."""
    L, nc, kappa = (8, 4, 4, 6), 3, 0.11
    tol = {q.HALF: 2e-3, q.BF16: 1.5e-2, q.DOUBLE: 1e-13}[prec]
    if kind != q.HOP_AUTO and prec == q.DOUBLE:
        pytest.skip("the direct tensor-core form is 16-bit only")
    gauge, dg = _setup(L, nc, m, kappa, 31)
    o = q.default_options()
    o.t_boundary = -1.0
    q.check(q.lib().qcuSetSolverOptions(ctypes.byref(o)))
    q.check(q.lib().qcuSetHopKernel(kind))
    rnd = (lambda a: a) if prec == q.DOUBLE else (lambda a: _round(a, prec))
    inp = F.to_mrhs(F.gaussian_fermions(L, nc, m, 32, parities=1)[:, 0])
    d_in = to_dev(inp, prec)
    for dagger in (0, 1):
        for parity in (0, 1):
            d_out = empty_dev(inp.shape, prec)
            q.check(q.lib().qcuDslashMrhsContext(d_out.data_ptr(), d_in.data_ptr(), parity, dagger, prec, None))
            sync()
            ref = oracle_lib.hop(rnd(inp), rnd(gauge), L, parity, bool(dagger), -1.0)
            got = from_dev(d_out)
            assert rel_err(got, ref) <= tol
            d_out2 = empty_dev(inp.shape, prec)
            q.check(q.lib().qcuDslashMrhsContext(d_out2.data_ptr(), d_in.data_ptr(), parity, dagger, prec, None))
            sync()
            assert np.array_equal(got, from_dev(d_out2))
    assert q.lib().qcuGetKernelError(1) == 0


@pytest.mark.parametrize("nc,m,flags", [
    (3, 12, [1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 0]),   # staged kernel: group 1 inactive
    (3, 16, [0, 0, 0, 0, 1, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0, 1]),   # groups 0 and 2 inactive
    (3, 7, [1, 1, 0, 1, 0, 0, 0]),                   # generic kernel, partial group 1 inactive
    (6, 8, [0, 0, 0, 0, 0, 1, 0, 0]),                # N = 6 kernel: group 0 inactive
])
@pytest.mark.parametrize("prec", [q.HALF, q.BF16])
def test_context_hop_skips_inactive_groups(oracle_lib, prec, nc, m, flags):
    """qcuDslashMrhsContextActive with the tensor-core hop: groups of 4 RHS whose flags are
    all 0 keep the output buffer's previous contents bit for bit, every other group is
    bit-identical to the hop without flags."""
    L, kappa = (8, 4, 4, 6), 0.11
    gauge, dg = _setup(L, nc, m, kappa, 33)
    o = q.default_options()
    o.t_boundary = -1.0
    q.check(q.lib().qcuSetSolverOptions(ctypes.byref(o)))
    q.check(q.lib().qcuSetHopKernel(q.HOP_MMA_LINK))
    try:
        inp = F.to_mrhs(F.gaussian_fermions(L, nc, m, 34, parities=1)[:, 0])
        old = F.to_mrhs(F.gaussian_fermions(L, nc, m, 35, parities=1)[:, 0])
        d_in = to_dev(inp, prec)
        d_act = torch.tensor(flags, dtype=torch.int32, device="cuda")
        for parity in (0, 1):
            d_full = empty_dev(inp.shape, prec)
            q.check(q.lib().qcuDslashMrhsContext(d_full.data_ptr(), d_in.data_ptr(), parity, 0, prec, None))
            d_out = to_dev(old, prec)
            q.check(q.lib().qcuDslashMrhsContextActive(d_out.data_ptr(), d_in.data_ptr(), parity, 0, prec,
                                                        d_act.data_ptr(), None))
            sync()
            full, got, before = from_dev(d_full), from_dev(d_out), from_dev(to_dev(old, prec))
            for g0 in range(0, m, 4):
                sl = slice(g0, min(g0 + 4, m))
                if any(flags[sl]):
                    assert np.array_equal(got[..., sl], full[..., sl]), (parity, g0)
                else:
                    assert np.array_equal(got[..., sl], before[..., sl]), (parity, g0)
    finally:
        q.lib().qcuSetHopKernel(q.HOP_AUTO)
    assert q.lib().qcuGetKernelError(1) == 0


def test_context_hop_with_half_the_groups_inactive_is_faster():
    """The cost of the skipped groups: FP16, 24^3 x 48, N = 3, m = 8, tensor-core hop, CUDA
    events over 20 launches after 3 warm-up; with group 1 (RHS 4-7) inactive the staged hop
    computes one tile per site instead of two (no projections, MMAs or stores for the
    inactive group; the bulk copies still move whole site blocks), so it must take
    measurably less time than with both groups live."""
    L, nc, m, kappa = (24, 24, 24, 48), 3, 8, 0.124
    init(L, nc, m)
    vh = F.half_volume(L)
    dg = torch.randn((4, 2, vh, nc, nc, 2), device="cuda", dtype=torch.float64)   # timing only
    q.lib().loadQcuGauge(dg.data_ptr(), q.DOUBLE)
    q.lib().getDslash(0, 1.0 / (2 * kappa) - 4.0)
    q.check()
    q.check(q.lib().qcuSetHopKernel(q.HOP_MMA_LINK))
    try:
        d_in = torch.randn((vh, 4, nc, m, 2), device="cuda").to(torch.float16)
        d_out = torch.empty_like(d_in)
        masks = {"all": [1] * 8, "half": [1, 1, 1, 1, 0, 0, 0, 0]}
        times = {}
        for name, fl in masks.items():
            act = torch.tensor(fl, dtype=torch.int32, device="cuda")
            for _ in range(3):
                q.check(q.lib().qcuDslashMrhsContextActive(d_out.data_ptr(), d_in.data_ptr(), 0, 0, q.HALF,
                                                            act.data_ptr(), None))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            for i in range(20):
                q.lib().qcuDslashMrhsContextActive(d_out.data_ptr(), d_in.data_ptr(), i & 1, 0, q.HALF,
                                                   act.data_ptr(), None)
            e1.record()
            torch.cuda.synchronize()
            q.check()
            times[name] = e0.elapsed_time(e1) / 20
        print("hop ms", times)
        # measured on B200: 151 vs 164 us; the copies, not the MMAs, set most of the time
        assert times["half"] <= 0.96 * times["all"], times
    finally:
        q.lib().qcuSetHopKernel(q.HOP_AUTO)


def test_mixed_solve_drops_converged_rhs_groups(oracle_lib):
    """Mixed FP16 solve with the tensor-core sloppy hop where one group of 4 RHS is
    converged from the start (zero sources, as when a batch is padded to a multiple of 4):
    the sloppy hops skip that group, its solutions are exactly 0, and the live RHS reach the
    FP64 true-residual tolerance as when solved next to live partners."""
    L, nc, m, kappa, tol = (8, 4, 4, 8), 3, 8, 0.11, 1e-10
    gauge, dg = _setup(L, nc, m, kappa, 71, kind="smooth")
    vh = F.half_volume(L)
    o = q.default_options()
    o.solver = q.SOLVER_MIXED
    o.sloppy_precision = q.HALF
    o.stop_true_residual = 1
    o.t_boundary = -1.0
    q.check(q.lib().qcuSetSolverOptions(ctypes.byref(o)))
    q.check(q.lib().qcuSetHopKernel(q.HOP_MMA_LINK))
    try:
        b_live = F.gaussian_fermions(L, nc, m, 72)
        runs = {}
        for name in ("padded", "live"):
            b = b_live.copy()
            if name == "padded":
                b[4:] = 0
            ins = [to_dev(b[j]) for j in range(m)]
            outs = [empty_dev((2, vh, 4, nc)) for _ in range(m)]
            for j in range(m):
                q.lib().pushBackFermions(outs[j].data_ptr(), ins[j].data_ptr())
            q.lib().qcuInvert(2000, tol)
            assert q.status() == q.SUCCESS, q.last_error()
            x = np.stack([from_dev(v) for v in outs])
            runs[name] = (b, x, q.solve_stats().iterations)
        b, x, it_padded = runs["padded"]
        assert np.all(x[4:] == 0)
        res = oracle_lib.mat(x[:4], gauge, L, kappa, t_sign=-1.0) - b[:4]
        rel = np.linalg.norm(res.reshape(4, -1), axis=1) / np.linalg.norm(b[:4].reshape(4, -1), axis=1)
        assert np.all(rel <= 2 * tol), rel
        # the live group alone needs no more iterations than next to live partners
        assert it_padded <= runs["live"][2] + 3, (it_padded, runs["live"][2])
    finally:
        q.lib().qcuSetHopKernel(q.HOP_AUTO)
    assert q.lib().qcuGetKernelError(1) == 0


@pytest.mark.parametrize("prec", [q.DOUBLE, q.HALF])
@pytest.mark.parametrize("form", [q.HOP_FORM_XPAY, q.HOP_FORM_SCHUR_R0, q.HOP_FORM_SCHUR_TS, q.HOP_FORM_SCHUR,
                                  q.HOP_FORM_RESID])
def test_context_hop_forms(oracle_lib, prec, form):
    """qcuDslashMrhsContextForm: the solver's fused hop epilogues (for FP16 the staged
    tensor-core kernel at m = 12) against the oracle hop on the same rounded inputs, with
    their per-RHS sums."""
    L, nc, m, kappa, a = (8, 4, 4, 6), 3, 12, 0.11, 0.0121
    gauge, dg = _setup(L, nc, m, kappa, 37)
    o = q.default_options()
    o.t_boundary = -1.0
    q.check(q.lib().qcuSetSolverOptions(ctypes.byref(o)))
    rnd = (lambda v: v) if prec == q.DOUBLE else (lambda v: _round(v, prec))
    inp = rnd(F.to_mrhs(F.gaussian_fermions(L, nc, m, 38, parities=1)[:, 0]))
    x = rnd(F.to_mrhs(F.gaussian_fermions(L, nc, m, 39, parities=1)[:, 0]))
    r0 = rnd(F.to_mrhs(F.gaussian_fermions(L, nc, m, 40, parities=1)[:, 0]))
    d_out = empty_dev(inp.shape, prec)
    d_in, d_x, d_r0 = to_dev(inp, prec), to_dev(x, prec), to_dev(r0, prec)   # alive until the kernel ran
    red = torch.zeros((2 * m, 2), dtype=torch.float64, device="cuda")
    q.check(q.lib().qcuDslashMrhsContextForm(d_out.data_ptr(), d_in.data_ptr(), d_x.data_ptr(), d_r0.data_ptr(), a,
                                             form, 1, prec, red.data_ptr(), None))
    sync()
    hop = oracle_lib.hop(inp, rnd(gauge), L, 1, False, -1.0)
    want = {q.HOP_FORM_XPAY: x + a * hop, q.HOP_FORM_RESID: r0 - (x - a * hop)}.get(form, x - a * hop)
    got = from_dev(d_out)
    tol = 1e-13 if prec == q.DOUBLE else 3e-3
    assert rel_err(got, want) <= tol
    sums = red.cpu().numpy()
    sums = sums[:, 0] + 1j * sums[:, 1]
    flat = lambda v: v.reshape(-1, m)
    stol = 1e-12 if prec == q.DOUBLE else 2e-3
    if form == q.HOP_FORM_SCHUR_R0:
        ref = np.sum(np.conj(flat(r0)) * flat(got), axis=0)
        assert np.allclose(sums[:m], ref, rtol=stol, atol=stol * np.abs(ref).max())
    elif form == q.HOP_FORM_SCHUR_TS:
        ref1 = np.sum(np.conj(flat(got)) * flat(x), axis=0)
        ref2 = np.sum(np.abs(flat(got)) ** 2, axis=0)
        assert np.allclose(sums[:m], ref1, rtol=stol, atol=stol * np.abs(ref1).max())
        assert np.allclose(sums[m:2 * m].real, ref2, rtol=stol)
    elif form == q.HOP_FORM_RESID:
        ref = np.sum(np.abs(flat(got)) ** 2, axis=0)
        assert np.allclose(sums[:m].real, ref, rtol=stol)
    assert q.lib().qcuGetKernelError(1) == 0


def test_staged_hop_bounded_wait_gives_up_with_an_error(oracle_lib):
    """The staged tensor-core hop's bounded waits: with its stages armed but never filled
    (qcuHopWaitSelfTest) every wait gives up after the given cycle count and the kernel ends
    with the device error flag set, instead of hanging; afterwards the flag is clear and the
    context's hop still matches the oracle."""
    L, nc, m, kappa = (8, 4, 4, 8), 3, 12, 0.11
    gauge, dg = _setup(L, nc, m, kappa, 91)
    o = q.default_options()
    o.t_boundary = -1.0
    q.check(q.lib().qcuSetSolverOptions(ctypes.byref(o)))
    q.check(q.lib().qcuSetHopKernel(q.HOP_MMA_LINK))
    timed_out = ctypes.c_int(0)
    q.check(q.lib().qcuHopWaitSelfTest(1 << 20, ctypes.byref(timed_out)))
    assert timed_out.value == 1
    assert q.lib().qcuGetKernelError(1) == 0
    inp = F.to_mrhs(F.gaussian_fermions(L, nc, m, 92, parities=1)[:, 0])
    d_in = to_dev(inp, q.HALF)
    d_out = empty_dev(inp.shape, q.HALF)
    q.check(q.lib().qcuDslashMrhsContext(d_out.data_ptr(), d_in.data_ptr(), 0, 0, q.HALF, None))
    sync()
    ref = oracle_lib.hop(_round(inp, q.HALF), _round(gauge, q.HALF), L, 0, False, -1.0)
    assert rel_err(from_dev(d_out), ref) <= 2e-3
    assert q.lib().qcuGetKernelError(1) == 0


def test_wait_self_test_rejects_unstaged_shapes():
    L, nc, m, kappa = (4, 4, 4, 4), 3, 6, 0.11
    _setup(L, nc, m, kappa, 93)
    timed_out = ctypes.c_int(0)
    assert q.lib().qcuHopWaitSelfTest(1 << 20, ctypes.byref(timed_out)) == q.ERR_UNSUPPORTED
    assert q.lib().qcuHopWaitSelfTest(0, ctypes.byref(timed_out)) == q.ERR_INVALID


_LAST = {"error": ""}


def _invert(L, nc, m, kappa, tol, seed, opts=None, max_iter=2000, kind="haar", t_boundary=1.0):
    gauge, dg = _setup(L, nc, m, kappa, seed, kind=kind)
    o = q.default_options()
    o.t_boundary = t_boundary
    if opts:
        for k, v in opts.items():
            setattr(o, k, v)
    q.check(q.lib().qcuSetSolverOptions(ctypes.byref(o)))
    vh = F.half_volume(L)
    b = F.gaussian_fermions(L, nc, m, seed + 1)
    ins = [to_dev(b[j]) for j in range(m)]
    outs = [empty_dev((2, vh, 4, nc)) for _ in range(m)]
    for j in range(m):
        q.lib().pushBackFermions(outs[j].data_ptr(), ins[j].data_ptr())
    q.lib().qcuInvert(max_iter, tol)
    st = q.status()
    _LAST["error"] = q.last_error()   # reading the statistics clears the message
    x = np.stack([from_dev(o) for o in outs])
    return gauge, b, x, st, q.solve_stats()


def test_repeated_solves_reuse_the_iteration_graph(oracle_lib):
    """Several qcuInvert calls on one context.  Each solve captures its block of iterations
    again and updates the executable graph the context keeps in place (cudaGraphExecUpdate),
    or instantiates anew when the update is refused.  The sequence covers both: FP64 with new
    sources (same topology: updated in place), FP64 with another check_interval and mixed
    FP16 (other topologies), mixed FP16 with the sloppy hop kernel forced to another kind
    (same topology, other kernel nodes), and FP64 again.  Every solution meets M x = b to the
    tolerance on the full system (oracle), and the iteration counts are plausible."""
    L, nc, m, kappa, tol = (8, 4, 4, 8), 3, 8, 0.11, 1e-10
    gauge, dg = _setup(L, nc, m, kappa, 41, kind="smooth")
    vh = F.half_volume(L)
    steps = [
        dict(solver=q.SOLVER_FUSED, check_interval=8, seed=42, kernel=q.HOP_AUTO),
        dict(solver=q.SOLVER_FUSED, check_interval=8, seed=43, kernel=q.HOP_AUTO),
        dict(solver=q.SOLVER_FUSED, check_interval=4, seed=44, kernel=q.HOP_AUTO),
        dict(solver=q.SOLVER_MIXED, check_interval=8, seed=45, kernel=q.HOP_AUTO),
        dict(solver=q.SOLVER_MIXED, check_interval=8, seed=46, kernel=q.HOP_PACKED16_PAIRS),
        dict(solver=q.SOLVER_MIXED, check_interval=8, seed=47, kernel=q.HOP_MMA_LINK),
        dict(solver=q.SOLVER_FUSED, check_interval=8, seed=48, kernel=q.HOP_AUTO),
    ]
    try:
        for i, stp in enumerate(steps):
            o = q.default_options()
            o.solver = stp["solver"]
            o.sloppy_precision = q.HALF
            o.check_interval = stp["check_interval"]
            o.stop_true_residual = 1
            o.t_boundary = -1.0
            q.check(q.lib().qcuSetSolverOptions(ctypes.byref(o)))
            q.check(q.lib().qcuSetHopKernel(stp["kernel"]))
            b = F.gaussian_fermions(L, nc, m, stp["seed"])
            ins = [to_dev(b[j]) for j in range(m)]
            outs = [empty_dev((2, vh, 4, nc)) for _ in range(m)]
            for j in range(m):
                q.lib().pushBackFermions(outs[j].data_ptr(), ins[j].data_ptr())
            q.lib().qcuInvert(2000, tol)
            assert q.status() == q.SUCCESS, f"solve {i}: {q.last_error()}"
            stats = q.solve_stats()
            assert 5 <= stats.iterations <= 200, f"solve {i}: {stats.iterations} iterations"
            x = np.stack([from_dev(v) for v in outs])
            res = oracle_lib.mat(x, gauge, L, kappa, t_sign=-1.0) - b
            rel = np.linalg.norm(res.reshape(m, -1), axis=1) / np.linalg.norm(b.reshape(m, -1), axis=1)
            assert np.all(rel <= 2 * tol), f"solve {i}: {rel.max()}"
    finally:
        q.lib().qcuSetHopKernel(q.HOP_AUTO)
    assert q.lib().qcuGetKernelError(1) == 0


def test_invert_matches_oracle_reference_rule(oracle_lib):
    """Config 1: 8^4, SU(3) Haar, m = 4, kappa = 0.10, antiperiodic t, tol 1e-10."""
    L, nc, m, kappa, tol = (8, 8, 8, 8), 3, 4, 0.10, 1e-10
    gauge, b, x, st, stats = _invert(L, nc, m, kappa, tol, 10, t_boundary=-1.0)
    assert st == q.SUCCESS, q.last_error()
    bm = np.stack([F.to_mrhs(b[:, 0]), F.to_mrhs(b[:, 1])])
    xo, it, rr = oracle_lib.bicgstab(bm, gauge, L, kappa, 2000, tol, t_sign=-1.0)
    assert abs(stats.iterations - it) <= 1
    xref = np.stack([F.from_mrhs(xo[0]), F.from_mrhs(xo[1])], axis=1)
    assert rel_err(x, xref) <= 1e-9
    res = oracle_lib.mat(x, gauge, L, kappa, t_sign=-1.0) - b
    true_rel = np.linalg.norm(res.reshape(m, -1), axis=1) / np.linalg.norm(b.reshape(m, -1), axis=1)
    assert np.allclose(true_rel, np.array(stats.true_residual[:m]), rtol=1e-3, atol=1e-14)
    assert np.all(np.array(stats.recursive_residual[:m]) <= tol)


def test_invert_true_residual_rule(oracle_lib):
    L, nc, m, kappa, tol = (8, 4, 4, 8), 3, 3, 0.12, 1e-10
    gauge, b, x, st, stats = _invert(L, nc, m, kappa, tol, 12, opts={"stop_true_residual": 1},
                                     kind="smooth")
    assert st == q.SUCCESS, q.last_error()
    res = oracle_lib.mat(x, gauge, L, kappa) - b
    true_rel = np.linalg.norm(res.reshape(m, -1), axis=1) / np.linalg.norm(b.reshape(m, -1), axis=1)
    assert np.all(true_rel <= 1.5 * tol)


@pytest.mark.parametrize("sloppy", [q.SINGLE, q.HALF, q.BF16])
def test_mixed_precision_reaches_fp64_true_residual(oracle_lib, sloppy):
    L, nc, m, kappa, tol = (8, 8, 8, 8), 3, 4, 0.124, 1e-10
    gauge, b, x, st, stats = _invert(L, nc, m, kappa, tol, 14, kind="smooth", t_boundary=-1.0,
                                     opts={"solver": q.SOLVER_MIXED, "sloppy_precision": sloppy})
    assert st == q.SUCCESS, q.last_error()
    assert stats.reliable_updates >= 1
    res = oracle_lib.mat(x, gauge, L, kappa, t_sign=-1.0) - b
    true_rel = np.linalg.norm(res.reshape(m, -1), axis=1) / np.linalg.norm(b.reshape(m, -1), axis=1)
    assert np.all(true_rel <= tol)
    assert np.allclose(true_rel, np.array(stats.true_residual[:m]), rtol=1e-2, atol=1e-15)


@pytest.mark.parametrize("kind", [q.HOP_PACKED16, q.HOP_PACKED16_ACC16, q.HOP_PACKED16_PAIRS, q.HOP_MMA_LINK],
                         ids=["packed16", "packed16_acc16", "packed16_pairs", "mma_link"])
@pytest.mark.parametrize("sloppy", [q.HALF, q.BF16])
def test_mixed_precision_with_packed_hop(oracle_lib, sloppy, kind):
    """The packed 16-bit hop inside the mixed solver: its Schur epilogues and fused
    reductions drive the sloppy iteration, FP64 reliable updates keep the true residual."""
    L, nc, m, kappa, tol = (8, 8, 8, 8), 3, 4, 0.124, 1e-10
    q.check(q.lib().qcuSetHopKernel(kind))
    try:
        gauge, b, x, st, stats = _invert(L, nc, m, kappa, tol, 15, kind="smooth", t_boundary=-1.0,
                                         opts={"solver": q.SOLVER_MIXED, "sloppy_precision": sloppy,
                                               "reliable_delta": 0.003})
    finally:
        q.lib().qcuSetHopKernel(q.HOP_AUTO)
    assert st == q.SUCCESS, q.last_error()
    res = oracle_lib.mat(x, gauge, L, kappa, t_sign=-1.0) - b
    true_rel = np.linalg.norm(res.reshape(m, -1), axis=1) / np.linalg.norm(b.reshape(m, -1), axis=1)
    assert np.all(true_rel <= tol)


@pytest.mark.parametrize("m", [8, 12])
@pytest.mark.parametrize("sloppy", [q.HALF, q.BF16])
def test_mixed_precision_two_rhs_kernel(oracle_lib, sloppy, m):
    """The product configuration of the mixed solver: SU(3) with an RHS count the two-RHS
    packed kernel takes, so every sloppy hop (plain, and the Schur forms that stage x and
    r0 in shared memory and reduce) runs in it.  Same convergence as with the one-RHS
    packed kernel (identical arithmetic per RHS) and the FP64 true residual."""
    L, nc, kappa, tol = (8, 8, 8, 8), 3, 0.124, 1e-10
    out = {}
    for kind in (q.HOP_PACKED16_PAIRS, q.HOP_PACKED16):
        q.check(q.lib().qcuSetHopKernel(kind))
        try:
            gauge, b, x, st, stats = _invert(L, nc, m, kappa, tol, 16, kind="smooth", t_boundary=-1.0,
                                             opts={"solver": q.SOLVER_MIXED, "sloppy_precision": sloppy,
                                                   "reliable_delta": 0.003})
        finally:
            q.lib().qcuSetHopKernel(q.HOP_AUTO)
        assert st == q.SUCCESS, _LAST["error"]
        res = oracle_lib.mat(x, gauge, L, kappa, t_sign=-1.0) - b
        true_rel = np.linalg.norm(res.reshape(m, -1), axis=1) / np.linalg.norm(b.reshape(m, -1), axis=1)
        assert np.all(true_rel <= tol)
        out[kind] = (x, stats.iterations)
    (xp, itp), (xg, itg) = out[q.HOP_PACKED16_PAIRS], out[q.HOP_PACKED16]
    assert abs(itp - itg) <= 2
    assert rel_err(xp, xg) <= 1e-9


@pytest.mark.parametrize("m", [8, 12, 16])
@pytest.mark.parametrize("sloppy", [q.HALF, q.BF16])
def test_mixed_precision_mma16_kernel(oracle_lib, sloppy, m):
    """The mixed solver with every sloppy hop (plain and the reducing Schur forms) in the
    warp-MMA kernel reaches the FP64 true residual and the solution of the two-RHS packed
    kernel (different rounding inside the hop, same converged solution)."""
    L, nc, kappa, tol = (8, 8, 8, 8), 3, 0.124, 1e-10
    out = {}
    for kind in (q.HOP_MMA16, q.HOP_PACKED16_PAIRS):
        q.check(q.lib().qcuSetHopKernel(kind))
        try:
            gauge, b, x, st, stats = _invert(L, nc, m, kappa, tol, 18, kind="smooth", t_boundary=-1.0,
                                             opts={"solver": q.SOLVER_MIXED, "sloppy_precision": sloppy,
                                                   "reliable_delta": 0.003})
        finally:
            q.lib().qcuSetHopKernel(q.HOP_AUTO)
        assert st == q.SUCCESS, _LAST["error"]
        res = oracle_lib.mat(x, gauge, L, kappa, t_sign=-1.0) - b
        true_rel = np.linalg.norm(res.reshape(m, -1), axis=1) / np.linalg.norm(b.reshape(m, -1), axis=1)
        assert np.all(true_rel <= tol)
        out[kind] = (x, stats.iterations)
    xp, itp = out[q.HOP_PACKED16_PAIRS]
    for kind in (q.HOP_MMA16,):
        xm, itm = out[kind]
        assert abs(itm - itp) <= 0.25 * itp + 2
        assert rel_err(xm, xp) <= 1e-7


@pytest.mark.parametrize("quorum", [0.5, 1.0])
@pytest.mark.parametrize("sloppy", [q.HALF, q.BF16])
def test_mixed_precision_reliable_quorum(oracle_lib, sloppy, quorum):
    """reliable_quorum: the reliable update waits until that fraction of the unconverged
    RHS met the delta rule.  The solve still stops only on the FP64 true residual, and it
    needs about as many reliable updates as the any-RHS rule on the same system, or fewer."""
    L, nc, m, kappa, tol = (8, 8, 8, 8), 3, 8, 0.124, 1e-10
    updates = {}
    for qr in (0.0, quorum):
        gauge, b, x, st, stats = _invert(L, nc, m, kappa, tol, 17, kind="smooth", t_boundary=-1.0,
                                         opts={"solver": q.SOLVER_MIXED, "sloppy_precision": sloppy,
                                               "reliable_delta": 0.003, "reliable_quorum": qr})
        assert st == q.SUCCESS, _LAST["error"]
        res = oracle_lib.mat(x, gauge, L, kappa, t_sign=-1.0) - b
        true_rel = np.linalg.norm(res.reshape(m, -1), axis=1) / np.linalg.norm(b.reshape(m, -1), axis=1)
        assert np.all(true_rel <= tol)
        updates[qr] = stats.reliable_updates
    assert 1 <= updates[quorum] <= updates[0.0] + 1


@pytest.mark.parametrize("true_rule", [0, 1], ids=["schur_rule", "true_rule"])
def test_cgnr_matches_oracle(oracle_lib, true_rule):
    """QCU_SOLVER_CGNR: CG on A^dag A x = A^dag b' follows the oracle's CGNR iterate by
    iterate (same iteration count within one, same solution), meets its stopping rule,
    and reports the FP64 true residual the oracle recomputes; the solution agrees with
    the BiCGStab one."""
    L, nc, m, kappa, tol = (8, 8, 8, 8), 3, 4, 0.10, 1e-10
    gauge, b, x, st, stats = _invert(L, nc, m, kappa, tol, 30, t_boundary=-1.0,
                                     opts={"solver": q.SOLVER_CGNR, "stop_true_residual": true_rule})
    assert st == q.SUCCESS, q.last_error()
    bm = np.stack([F.to_mrhs(b[:, 0]), F.to_mrhs(b[:, 1])])
    xo, it, rr = oracle_lib.cgnr(bm, gauge, L, kappa, 2000, tol, t_sign=-1.0, true_rule=bool(true_rule))
    assert it > 0 and abs(stats.iterations - it) <= 1
    xref = np.stack([F.from_mrhs(xo[0]), F.from_mrhs(xo[1])], axis=1)
    assert rel_err(x, xref) <= 1e-8
    assert np.all(np.array(stats.recursive_residual[:m]) <= tol)
    res = oracle_lib.mat(x, gauge, L, kappa, t_sign=-1.0) - b
    true_rel = np.linalg.norm(res.reshape(m, -1), axis=1) / np.linalg.norm(b.reshape(m, -1), axis=1)
    assert np.all(true_rel <= 10 * tol)
    assert np.allclose(true_rel, np.array(stats.true_residual[:m]), rtol=1e-2, atol=1e-14)
    xb, itb, _ = oracle_lib.bicgstab(bm, gauge, L, kappa, 2000, tol, t_sign=-1.0)
    xbr = np.stack([F.from_mrhs(xb[0]), F.from_mrhs(xb[1])], axis=1)
    assert rel_err(x, xbr) <= 1e-8


def test_cgnr_single_precision(oracle_lib):
    """FP32 fields through CGNR: converges to the FP32-reachable tolerance."""
    L, nc, m, kappa, tol = (8, 4, 4, 8), 3, 3, 0.12, 1e-5
    init(L, nc, m, q.SINGLE, q.SINGLE)
    gauge = F.gauge_field(L, nc, 31, kind="smooth", eps=0.3)
    dg = to_dev(gauge, q.SINGLE)
    q.lib().loadQcuGauge(dg.data_ptr(), q.SINGLE)
    q.lib().getDslash(0, 1.0 / (2 * kappa) - 4.0)
    o = q.default_options()
    o.solver = q.SOLVER_CGNR
    q.check(q.lib().qcuSetSolverOptions(ctypes.byref(o)))
    vh = F.half_volume(L)
    b = F.gaussian_fermions(L, nc, m, 32)
    ins = [to_dev(b[j], q.SINGLE) for j in range(m)]
    outs = [empty_dev((2, vh, 4, nc), q.SINGLE) for _ in range(m)]
    for j in range(m):
        q.lib().pushBackFermions(outs[j].data_ptr(), ins[j].data_ptr())
    q.lib().qcuInvert(2000, tol)
    assert q.status() == q.SUCCESS, q.last_error()
    x = np.stack([from_dev(t) for t in outs])
    b32 = np.stack([from_dev(t) for t in ins])
    res = oracle_lib.mat(x, gauge, L, kappa) - b32
    true_rel = np.linalg.norm(res.reshape(m, -1), axis=1) / np.linalg.norm(b32.reshape(m, -1), axis=1)
    assert np.all(true_rel <= 10 * tol)


def test_cgnr_not_converged_and_options():
    L, nc, m, kappa = (4, 4, 4, 4), 3, 2, 0.12
    _, _, _, st, stats = _invert(L, nc, m, kappa, 1e-12, 40, max_iter=3, opts={"solver": q.SOLVER_CGNR})
    assert st == q.ERR_NOT_CONVERGED
    assert stats.iterations == 3
    o = q.default_options()
    o.solver = q.SOLVER_CGNR + 1
    assert q.lib().qcuSetSolverOptions(ctypes.byref(o)) == q.ERR_INVALID
    o.solver = q.SOLVER_CGNR
    init(L, nc, m, q.HALF, q.HALF)
    assert q.lib().qcuSetSolverOptions(ctypes.byref(o)) == q.SUCCESS


@pytest.mark.parametrize("sloppy", [q.SINGLE, q.HALF])
def test_mixed_precision_stops_when_the_residual_stagnates(oracle_lib, sloppy):
    """A tolerance below FP64 reach: the FP64 residual stops falling, and the mixed solver
    ends as not converged after the stall limit (32 reliable updates without a 2% gain)
    instead of iterating to max_iteration; x is finite and as good as FP64 allows."""
    L, nc, m, kappa = (8, 8, 8, 8), 3, 4, 0.12
    gauge, b, x, st, stats = _invert(L, nc, m, kappa, 1e-17, 17, max_iter=5000, kind="smooth",
                                     t_boundary=-1.0,
                                     opts={"solver": q.SOLVER_MIXED, "sloppy_precision": sloppy,
                                           "reliable_delta": 0.1})
    assert st == q.ERR_NOT_CONVERGED
    assert "stagnated" in _LAST["error"]
    assert stats.iterations < 5000
    assert stats.reliable_updates >= 32
    res = oracle_lib.mat(x, gauge, L, kappa, t_sign=-1.0) - b
    true_rel = np.linalg.norm(res.reshape(m, -1), axis=1) / np.linalg.norm(b.reshape(m, -1), axis=1)
    assert np.all(np.isfinite(x)) and np.all(true_rel <= 1e-13)


def test_invert_not_converged_status():
    L, nc, m = (4, 4, 4, 4), 3, 2
    gauge, b, x, st, stats = _invert(L, nc, m, 0.12, 1e-14, 16, max_iter=3)
    assert st == q.ERR_NOT_CONVERGED
    assert stats.iterations == 3
    assert np.all(np.isfinite(x))


def test_zero_source_rhs_gives_zero_solution(oracle_lib):
    L, nc, m, kappa = (4, 4, 4, 4), 3, 3, 0.1
    gauge, dg = _setup(L, nc, m, kappa, 18)
    vh = F.half_volume(L)
    b = F.gaussian_fermions(L, nc, m, 19)
    b[1] = 0
    ins = [to_dev(b[j]) for j in range(m)]
    outs = [empty_dev((2, vh, 4, nc)) for _ in range(m)]
    for j in range(m):
        q.lib().pushBackFermions(outs[j].data_ptr(), ins[j].data_ptr())
    q.lib().qcuInvert(500, 1e-10)
    assert q.status() == q.SUCCESS, q.last_error()
    x = np.stack([from_dev(o) for o in outs])
    assert np.all(x[1] == 0)
    res = oracle_lib.mat(x, gauge, L, kappa) - b
    assert np.linalg.norm(res[0]) / np.linalg.norm(b[0]) < 1e-9


def test_queue_rules():
    L, nc, m = (4, 4, 4, 4), 3, 2
    _setup(L, nc, m, 0.1, 20)
    d = empty_dev((2, F.half_volume(L), 4, nc))
    q.lib().pushBackFermions(d.data_ptr(), d.data_ptr())
    q.lib().start_dslash(0, 0)
    assert q.status() == q.ERR_STATE          # queue not full
    q.lib().pushBackFermions(d.data_ptr(), d.data_ptr())
    q.lib().pushBackFermions(d.data_ptr(), d.data_ptr())
    q.lib().pushBackFermions(d.data_ptr(), d.data_ptr())
    assert q.status() == q.ERR_STATE          # queue full
    q.lib().getDslash(1, 0.0)
    assert q.status() == q.ERR_UNSUPPORTED    # only Wilson


def test_gauge_eo_precondition_through_context(oracle_lib):
    L, nc, m = (4, 2, 2, 6), 3, 1
    init(L, nc, m)
    V = 4 * 2 * 2 * 6
    rng = np.random.default_rng(21)
    lex = rng.standard_normal((4, V, nc, nc)) + 1j * rng.standard_normal((4, V, nc, nc))
    dl = to_dev(lex)
    de = empty_dev(lex.shape)
    q.lib().gauge_eo_precondition(de.data_ptr(), dl.data_ptr(), q.DOUBLE)
    q.check()
    assert np.array_equal(from_dev(de), oracle_lib.gauge_to_eo(lex, L))
    back = empty_dev(lex.shape)
    q.lib().gauge_reverse_eo_precondition(back.data_ptr(), de.data_ptr(), q.DOUBLE)
    q.check()
    assert np.array_equal(from_dev(back), lex)
