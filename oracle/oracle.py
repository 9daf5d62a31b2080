"""ctypes binding of the CPU oracle (oracle/libqcu_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, always as the checker or the timed CPU
baseline, never as part of the product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libqcu_oracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        l = ctypes.CDLL(_LIB_PATH)
        l.oracle_hop_mrhs.argtypes = [_dp, _dp, _dp, _ip, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_double]
        l.oracle_gather.argtypes = [_dp, _dp, ctypes.c_long, ctypes.c_int, ctypes.c_int]
        l.oracle_scatter.argtypes = [_dp, _dp, ctypes.c_long, ctypes.c_int, ctypes.c_int]
        l.oracle_mat.argtypes = [_dp, _dp, _dp, _ip, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                 ctypes.c_int, ctypes.c_double]
        l.oracle_schur.argtypes = [_dp, _dp, _dp, _dp, _ip, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_double, ctypes.c_double]
        for name in ("oracle_dotc",):
            getattr(l, name).argtypes = [_dp, _dp, _dp, ctypes.c_long, ctypes.c_int]
        l.oracle_norm.argtypes = [_dp, _dp, ctypes.c_long, ctypes.c_int]
        for name in ("oracle_xsay", "oracle_xpay"):
            getattr(l, name).argtypes = [_dp, _dp, _dp, _dp, ctypes.c_long, ctypes.c_int]
        l.oracle_axpby.argtypes = [_dp, _dp, _dp, _dp, _dp, ctypes.c_long, ctypes.c_int]
        l.oracle_axpbypcz.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, _dp, ctypes.c_long, ctypes.c_int]
        l.oracle_bicgstab.argtypes = [_dp, _dp, _dp, _ip, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_int, ctypes.c_double, _dp]
        l.oracle_bicgstab.restype = ctypes.c_int
        for name in ("oracle_gauge_to_eo", "oracle_gauge_from_eo", "oracle_fermion_to_eo",
                     "oracle_fermion_from_eo"):
            getattr(l, name).argtypes = [_dp, _dp, _ip, ctypes.c_int]
        for name in ("oracle_ptc_forward", "oracle_ptc_adjoint", "oracle_ptc_wgrad"):
            getattr(l, name).argtypes = [_dp, _dp, _dp, _dp, _ip, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_double]
        l.oracle_set_threads.argtypes = [ctypes.c_int]
        l.oracle_get_threads.restype = ctypes.c_int
        _lib = l
    return _lib


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    assert a.dtype in (np.complex128, np.float64)
    return a.ctypes.data_as(_dp)


def _L(L):
    return (ctypes.c_int * 4)(*[int(v) for v in L])


def _c(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def get_threads() -> int:
    return int(lib().oracle_get_threads())


def hop(in_mrhs, gauge, L, parity, dagger=False, t_sign=1.0):
    """D_p on the gathered layout: in [Vh][4][N][m] (parity 1-p) -> out (parity p)."""
    in_mrhs = _c(in_mrhs)
    gauge = _c(gauge)
    nc, m = in_mrhs.shape[2], in_mrhs.shape[3]
    out = np.empty_like(in_mrhs)
    lib().oracle_hop_mrhs(_ptr(out), _ptr(in_mrhs), _ptr(gauge), _L(L), nc, m, int(parity),
                          int(bool(dagger)), float(t_sign))
    return out


def mat(fermions, gauge, L, kappa, dagger=False, t_sign=1.0):
    """M = 1 - kappa D on per-RHS EO fields [m][2][Vh][4][N]."""
    fermions = _c(fermions)
    gauge = _c(gauge)
    m, nc = fermions.shape[0], fermions.shape[4]
    out = np.empty_like(fermions)
    lib().oracle_mat(_ptr(out), _ptr(fermions), _ptr(gauge), _L(L), nc, m, float(kappa),
                     int(bool(dagger)), float(t_sign))
    return out


def schur(in_odd, gauge, L, kappa, t_sign=1.0):
    in_odd = _c(in_odd)
    gauge = _c(gauge)
    nc, m = in_odd.shape[2], in_odd.shape[3]
    out = np.empty_like(in_odd)
    tmp = np.empty_like(in_odd)
    lib().oracle_schur(_ptr(out), _ptr(in_odd), _ptr(tmp), _ptr(gauge), _L(L), nc, m, float(kappa),
                       float(t_sign))
    return out


def dotc(a, b, m):
    a = _c(a); b = _c(b)
    res = np.empty(m, dtype=np.complex128)
    lib().oracle_dotc(_ptr(res), _ptr(a), _ptr(b), a.size // m, m)
    return res


def norm(a, m):
    a = _c(a)
    res = np.empty(m, dtype=np.float64)
    lib().oracle_norm(_ptr(res), _ptr(a), a.size // m, m)
    return res


def xsay(x, a, y, m):
    x = _c(x); a = _c(a); y = _c(y)
    res = np.empty_like(x)
    lib().oracle_xsay(_ptr(res), _ptr(x), _ptr(a), _ptr(y), x.size // m, m)
    return res


def xpay(x, a, y, m):
    x = _c(x); a = _c(a); y = _c(y)
    res = np.empty_like(x)
    lib().oracle_xpay(_ptr(res), _ptr(x), _ptr(a), _ptr(y), x.size // m, m)
    return res


def axpby(a, x, b, y, m):
    a = _c(a); x = _c(x); b = _c(b); y = _c(y)
    res = np.empty_like(x)
    lib().oracle_axpby(_ptr(res), _ptr(a), _ptr(x), _ptr(b), _ptr(y), x.size // m, m)
    return res


def axpbypcz(a, x, b, y, c, z, m):
    a = _c(a); x = _c(x); b = _c(b); y = _c(y); c = _c(c); z = _c(z)
    res = np.empty_like(x)
    lib().oracle_axpbypcz(_ptr(res), _ptr(a), _ptr(x), _ptr(b), _ptr(y), _ptr(c), _ptr(z),
                          x.size // m, m)
    return res


def bicgstab(b_mrhs_full, gauge, L, kappa, max_iter, tol, t_sign=1.0):
    """Schur BiCGStab policy 1. b: gathered full lattice [2][Vh][4][N][m].
    Returns (x, iterations or -1, per-RHS recursive relative residual)."""
    b = _c(b_mrhs_full)
    gauge = _c(gauge)
    nc, m = b.shape[3], b.shape[4]
    x = np.zeros_like(b)
    rr = np.empty(m, dtype=np.float64)
    it = lib().oracle_bicgstab(_ptr(x), _ptr(b), _ptr(gauge), _L(L), nc, m, float(kappa),
                               float(t_sign), int(max_iter), float(tol), _ptr(rr))
    return x, int(it), rr


def cgnr(b_mrhs_full, gauge, L, kappa, max_iter, tol, t_sign=1.0, true_rule=False):
    """CG on the normal equations of the Schur system, A^dag A x_o = A^dag b'_o, with
    A = 1 - kappa^2 D_oe D_eo and A^dag from the dagger hops; per-RHS alpha and beta.
    Stops when every RHS has ||b' - A x_o|| <= tol ||b'|| (||b|| of the full system with
    true_rule).  The reference has no normal-equation solver: this restates textbook CGNR
    on the reference's hop (oracle_hop_mrhs) as the checker of the library's
    QCU_SOLVER_CGNR.  b: gathered full lattice [2][Vh][4][N][m].
    Returns (x, iterations or -1, per-RHS ||b' - A x_o|| / reference norm)."""
    b = _c(b_mrhs_full)
    m = b.shape[4]
    k2 = kappa * kappa

    def op(v, dag):
        t = hop(v, gauge, L, 0, dag, t_sign)
        return v - k2 * hop(t, gauge, L, 1, dag, t_sign)

    def dot(a, c):
        return np.einsum("vsci,vsci->i", a.conj(), c).real

    be, bo = b[0], b[1]
    bp = bo + kappa * hop(be, gauge, L, 1, False, t_sign)
    ref = dot(be, be) + dot(bo, bo) if true_rule else dot(bp, bp)
    x = np.zeros_like(bp)
    s = bp.copy()
    r = op(bp, True)
    p = r.copy()
    rr = dot(r, r)
    it = 0
    ss = dot(s, s)
    while not np.all(ss <= tol * tol * ref):
        if it >= max_iter:
            it = -1
            break
        q = op(p, False)
        z = op(q, True)
        qq = dot(q, q)
        alpha = np.where(qq > 0, rr / np.where(qq > 0, qq, 1.0), 0.0)
        x = x + alpha * p
        s = s - alpha * q
        r = r - alpha * z
        rrn = dot(r, r)
        beta = np.where(rr > 0, rrn / np.where(rr > 0, rr, 1.0), 0.0)
        rr = rrn
        p = r + beta * p
        ss = dot(s, s)
        it += 1
    xe = be + kappa * hop(x, gauge, L, 0, False, t_sign)
    rel = np.sqrt(ss / np.where(ref > 0, ref, 1.0))
    return np.stack([xe, x]), it, rel


def gauge_to_eo(lex, L):
    lex = _c(lex)
    nc = lex.shape[-1]
    eo = np.empty_like(lex)
    lib().oracle_gauge_to_eo(_ptr(eo), _ptr(lex), _L(L), nc)
    return eo


def gauge_from_eo(eo, L):
    eo = _c(eo)
    nc = eo.shape[-1]
    lex = np.empty_like(eo)
    lib().oracle_gauge_from_eo(_ptr(lex), _ptr(eo), _L(L), nc)
    return lex


def fermion_to_eo(lex, L):
    lex = _c(lex)
    nc = lex.shape[-1]
    eo = np.empty_like(lex)
    lib().oracle_fermion_to_eo(_ptr(eo), _ptr(lex), _L(L), nc)
    return eo


def fermion_from_eo(eo, L):
    eo = _c(eo)
    nc = eo.shape[-1]
    lex = np.empty_like(eo)
    lib().oracle_fermion_from_eo(_ptr(lex), _ptr(eo), _L(L), nc)
    return lex


# ---------------- learned preconditioner (parallel-transport convolution net) ----------------

def ptc_forward(inp, w, gauge, L, t_sign=1.0):
    """One layer: inp [cin][2][Vh][4][N][m], w [cout][cin][9][4][4] -> [cout][2][Vh][4][N][m]."""
    inp = _c(inp); w = _c(w); gauge = _c(gauge)
    cin, nc, m = inp.shape[0], inp.shape[4], inp.shape[5]
    cout = w.shape[0]
    assert w.shape[1] == cin
    out = np.empty((cout,) + inp.shape[1:], dtype=np.complex128)
    lib().oracle_ptc_forward(_ptr(out), _ptr(inp), _ptr(w), _ptr(gauge), _L(L), nc, m, cin, cout, float(t_sign))
    return out


def ptc_adjoint(gout, w, gauge, L, t_sign=1.0):
    """Adjoint of one layer: gout [cout][...] -> gin [cin][...]."""
    gout = _c(gout); w = _c(w); gauge = _c(gauge)
    cout, cin = w.shape[0], w.shape[1]
    nc, m = gout.shape[4], gout.shape[5]
    gin = np.empty((cin,) + gout.shape[1:], dtype=np.complex128)
    lib().oracle_ptc_adjoint(_ptr(gin), _ptr(gout), _ptr(w), _ptr(gauge), _L(L), nc, m, cin, cout, float(t_sign))
    return gin


def ptc_wgrad(gout, inp, gauge, L, t_sign=1.0):
    """Complex weight gradient tensor gw[cout][cin][9][4][4] of one layer."""
    gout = _c(gout); inp = _c(inp); gauge = _c(gauge)
    cout, cin = gout.shape[0], inp.shape[0]
    nc, m = inp.shape[4], inp.shape[5]
    gw = np.empty((cout, cin, 9, 4, 4), dtype=np.complex128)
    lib().oracle_ptc_wgrad(_ptr(gw), _ptr(gout), _ptr(inp), _ptr(gauge), _L(L), nc, m, cin, cout, float(t_sign))
    return gw


def _full_to_per_rhs(v):
    """gathered full lattice [2][Vh][4][N][m] -> per-RHS [m][2][Vh][4][N]"""
    return np.ascontiguousarray(np.moveaxis(v, -1, 0))


def _per_rhs_to_full(v):
    return np.ascontiguousarray(np.moveaxis(v, 0, -1))


def precond_apply(b, weights, gauge, L, t_sign=1.0):
    """P b for the layer stack `weights` (list of [cout][cin][9][4][4]); b [2][Vh][4][N][m]."""
    a = _c(b)[None]
    for w in weights:
        a = ptc_forward(a, w, gauge, L, t_sign)
    return a[0]


def precond_loss_grad(b, weights, gauge, L, kappa, t_sign=1.0):
    """Loss sum_j ||M P b_j - b_j||^2 / ||b_j||^2 and its gradient with respect to the real
    and imaginary parts of every weight (list of complex arrays: grad = dL/dRe + i dL/dIm)."""
    b = _c(b)
    acts = [b[None]]
    for w in weights:
        acts.append(ptc_forward(acts[-1], w, gauge, L, t_sign))
    y = acts[-1][0]
    r = _per_rhs_to_full(mat(_full_to_per_rhs(y), gauge, L, kappa, False, t_sign)) - b
    bn2 = np.sum(np.abs(b) ** 2, axis=(0, 1, 2, 3))
    loss = float(np.sum(np.sum(np.abs(r) ** 2, axis=(0, 1, 2, 3)) / bn2))
    g = _per_rhs_to_full(mat(_full_to_per_rhs(r), gauge, L, kappa, True, t_sign)) / bn2
    g = g[None]
    grads = [None] * len(weights)
    for li in range(len(weights) - 1, -1, -1):
        gw = ptc_wgrad(g, acts[li], gauge, L, t_sign)
        grads[li] = 2.0 * gw
        if li > 0:
            g = ptc_adjoint(g, weights[li], gauge, L, t_sign)
    return loss, grads
