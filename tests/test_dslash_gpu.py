"""Hop term on the GPU vs the CPU oracle, through the C ABI (qcuDslashMrhs & co.).

Tolerances (relative Frobenius error of the whole output):
  FP64 <= 1e-13 against the oracle on the same inputs;
  FP32 / FP16 / BF16 against the oracle run on the same *rounded* inputs:
  FP32 1e-6, FP16 2e-3, BF16 1.5e-2 (output rounding plus FP32 accumulation).
"""
import numpy as np
import pytest

import qcu_mrhs_b200 as q
from qcu_mrhs_b200 import fields as F
from tests.helpers import empty_dev, from_dev, rel_err, sync, to_dev

pytestmark = pytest.mark.gpu

TOL = {q.DOUBLE: 1e-13, q.SINGLE: 1e-6, q.HALF: 2e-3, q.BF16: 1.5e-2}


def _round(arr, prec):
    """Round a complex array to the storage precision and back (numpy/torch on CPU)."""
    import torch
    if prec == q.DOUBLE:
        return arr
    dt = {q.SINGLE: torch.float32, q.HALF: torch.float16, q.BF16: torch.bfloat16}[prec]
    a = np.ascontiguousarray(arr, dtype=np.complex128)
    t = torch.from_numpy(a.view(np.float64).reshape(a.shape + (2,)).copy()).to(dt).to(torch.float64).numpy()
    return t[..., 0] + 1j * t[..., 1]


def _problem(L, nc, m, seed, kind="haar"):
    gauge = F.gauge_field(L, nc, seed, kind=kind)
    psi = F.gaussian_fermions(L, nc, m, seed + 1, parities=1)[:, 0]
    return gauge, F.to_mrhs(psi)


def _hop_gpu(inp, gauge, L, parity, dagger, t_sign, prec):
    nc, m = inp.shape[2], inp.shape[3]
    d_in, d_g = to_dev(inp, prec), to_dev(gauge, prec)
    d_out = empty_dev(inp.shape, prec)
    rc = q.lib().qcuDslashMrhs(d_out.data_ptr(), d_in.data_ptr(), d_g.data_ptr(), q.lattice(L), nc, m,
                               parity, int(dagger), float(t_sign), prec, None)
    q.check(rc)
    sync()
    return from_dev(d_out)


@pytest.mark.parametrize("parity", [0, 1])
@pytest.mark.parametrize("dagger", [False, True])
@pytest.mark.parametrize("t_sign", [1.0, -1.0])
def test_fp64_hop_config1(oracle_lib, parity, dagger, t_sign):
    L, nc, m = (8, 8, 8, 8), 3, 4
    gauge, inp = _problem(L, nc, m, 11)
    ref = oracle_lib.hop(inp, gauge, L, parity, dagger, t_sign)
    got = _hop_gpu(inp, gauge, L, parity, dagger, t_sign, q.DOUBLE)
    assert rel_err(got, ref) <= TOL[q.DOUBLE]


@pytest.mark.parametrize("nc", [2, 3, 4, 5, 6, 7, 8])
@pytest.mark.parametrize("m", [1, 3, 12, 32])
def test_fp64_hop_colours_and_rhs(oracle_lib, nc, m):
    L = (4, 4, 2, 6)
    gauge, inp = _problem(L, nc, m, 20 + nc)
    for parity in (0, 1):
        ref = oracle_lib.hop(inp, gauge, L, parity, False, -1.0)
        got = _hop_gpu(inp, gauge, L, parity, False, -1.0, q.DOUBLE)
        assert rel_err(got, ref) <= TOL[q.DOUBLE]


@pytest.mark.parametrize("L", [(2, 2, 2, 2), (2, 4, 6, 2), (10, 2, 2, 4), (6, 6, 6, 6)])
def test_fp64_hop_shapes(oracle_lib, L):
    gauge, inp = _problem(L, 3, 5, 31)
    for parity in (0, 1):
        ref = oracle_lib.hop(inp, gauge, L, parity, True, -1.0)
        got = _hop_gpu(inp, gauge, L, parity, True, -1.0, q.DOUBLE)
        assert rel_err(got, ref) <= TOL[q.DOUBLE]


def test_fp64_hop_max_rhs(oracle_lib):
    L = (4, 2, 2, 4)
    gauge, inp = _problem(L, 3, 64, 33)
    ref = oracle_lib.hop(inp, gauge, L, 1, False, 1.0)
    assert rel_err(_hop_gpu(inp, gauge, L, 1, False, 1.0, q.DOUBLE), ref) <= TOL[q.DOUBLE]


@pytest.fixture
def hop_kernel(request):
    """Select the FP16/BF16 hop implementation for one test, restore AUTO afterwards."""
    q.check(q.lib().qcuSetHopKernel(request.param))
    yield request.param
    q.lib().qcuSetHopKernel(q.HOP_AUTO)


def _acc16_factor(kind, prec):
    """FP16 accumulation of the 8 hops (PACKED16_ACC16, FP16 storage only) adds about one
    FP16 rounding per hop: its tolerance is twice the FP16 one."""
    return 2.0 if (kind == q.HOP_PACKED16_ACC16 and prec == q.HALF) else 1.0


LOWP_KERNELS = [q.HOP_SIMT, q.HOP_SIMT_CS, q.HOP_TENSOR, q.HOP_PACKED16, q.HOP_PACKED16_ACC16,
                q.HOP_PACKED16_STAGED, q.HOP_PACKED16_PAIRS, q.HOP_MMA16, q.HOP_MMA_LINK, q.HOP_MMA_LINK_DIRECT]
LOWP_IDS = ["simt", "simt_cs", "tcgen05", "packed16", "packed16_acc16", "packed16_staged", "packed16_pairs", "mma16",
            "mma_link", "mma_link_direct"]


@pytest.mark.parametrize("hop_kernel", LOWP_KERNELS, indirect=True, ids=LOWP_IDS)
@pytest.mark.parametrize("prec", [q.SINGLE, q.HALF, q.BF16])
@pytest.mark.parametrize("nc,m", [(3, 4), (3, 12), (4, 8), (2, 32), (3, 17), (8, 16), (6, 5), (3, 1), (3, 8), (3, 16)])
def test_low_precision_hop(oracle_lib, prec, nc, m, hop_kernel):
    L = (8, 4, 4, 4)
    gauge, inp = _problem(L, nc, m, 40 + nc)
    gr, ir = _round(gauge, prec), _round(inp, prec)
    tol = TOL[prec] * _acc16_factor(hop_kernel, prec)
    for parity in (0, 1):
        for dagger in (False, True):
            ref = oracle_lib.hop(ir, gr, L, parity, dagger, -1.0)
            got = _hop_gpu(inp, gauge, L, parity, dagger, -1.0, prec)
            assert rel_err(got, ref) <= tol
            # error against the unrounded FP64 oracle stays within a few storage ulps
            ref64 = oracle_lib.hop(inp, gauge, L, parity, dagger, -1.0)
            assert rel_err(got, ref64) <= 4 * tol
    assert q.lib().qcuGetKernelError(1) == 0


@pytest.mark.parametrize("hop_kernel", [q.HOP_TENSOR, q.HOP_PACKED16, q.HOP_PACKED16_ACC16, q.HOP_PACKED16_STAGED,
                                        q.HOP_PACKED16_PAIRS, q.HOP_MMA_LINK], indirect=True,
                         ids=["tcgen05", "packed16", "packed16_acc16", "packed16_staged", "packed16_pairs",
                              "mma_link"])
@pytest.mark.parametrize("prec", [q.HALF, q.BF16])
@pytest.mark.parametrize("L", [(2, 2, 2, 2), (6, 2, 4, 2), (4, 4, 4, 6), (8, 8, 8, 10)])
def test_low_precision_hop_shapes_and_epilogues(oracle_lib, prec, L, hop_kernel):
    """Odd half volumes (last tile / staging pass holds one site), tiny lattices, several
    staging passes per block, xpay and Schur epilogues."""
    nc, m = 3, 7
    gauge, inp = _problem(L, nc, m, 70)
    gr, ir = _round(gauge, prec), _round(inp, prec)
    x = F.to_mrhs(F.gaussian_fermions(L, nc, m, 71, parities=1)[:, 0])
    xr = _round(x, prec)
    d_in, d_g, d_x = to_dev(inp, prec), to_dev(gauge, prec), to_dev(x, prec)
    d_out, d_tmp = empty_dev(inp.shape, prec), empty_dev(inp.shape, prec)
    tol = TOL[prec] * _acc16_factor(hop_kernel, prec)
    rc = q.lib().qcuDslashMrhsXpay(d_out.data_ptr(), d_in.data_ptr(), d_g.data_ptr(), d_x.data_ptr(), -0.37,
                                   q.lattice(L), nc, m, 1, 0, 1.0, prec, None)
    q.check(rc)
    sync()
    ref = xr - 0.37 * oracle_lib.hop(ir, gr, L, 1, False, 1.0)
    assert rel_err(from_dev(d_out), ref) <= tol
    rc = q.lib().qcuSchurMrhs(d_out.data_ptr(), d_in.data_ptr(), d_tmp.data_ptr(), d_g.data_ptr(), 0.11,
                              q.lattice(L), nc, m, -1.0, prec, None)
    q.check(rc)
    sync()
    ref = oracle_lib.schur(ir, gr, L, 0.11, -1.0)
    assert rel_err(from_dev(d_out), ref) <= 2 * tol
    assert q.lib().qcuGetKernelError(1) == 0


@pytest.mark.parametrize("hop_kernel", [q.HOP_MMA16], indirect=True, ids=["mma16"])
@pytest.mark.parametrize("prec", [q.HALF, q.BF16])
@pytest.mark.parametrize("m", [8, 12, 16])
@pytest.mark.parametrize("L", [(2, 2, 2, 2), (6, 2, 4, 2), (8, 4, 4, 8)])
def test_mma16_hop_shapes_and_epilogues(oracle_lib, prec, m, L, hop_kernel):
    """The warp-MMA hop (one warp per site, FP32 accumulation in the tensor cores) at the RHS
    counts it covers: both parities with and without dagger against the oracle on the same
    rounded inputs, odd half volumes, tiny lattices, the xpay and Schur epilogues."""
    nc = 3
    gauge, inp = _problem(L, nc, m, 80 + m)
    gr, ir = _round(gauge, prec), _round(inp, prec)
    tol = TOL[prec]
    for parity in (0, 1):
        for dagger in (False, True):
            ref = oracle_lib.hop(ir, gr, L, parity, dagger, -1.0)
            got = _hop_gpu(inp, gauge, L, parity, dagger, -1.0, prec)
            assert rel_err(got, ref) <= tol
    x = F.to_mrhs(F.gaussian_fermions(L, nc, m, 81, parities=1)[:, 0])
    xr = _round(x, prec)
    d_in, d_g, d_x = to_dev(inp, prec), to_dev(gauge, prec), to_dev(x, prec)
    d_out, d_tmp = empty_dev(inp.shape, prec), empty_dev(inp.shape, prec)
    q.check(q.lib().qcuDslashMrhsXpay(d_out.data_ptr(), d_in.data_ptr(), d_g.data_ptr(), d_x.data_ptr(), -0.37,
                                      q.lattice(L), nc, m, 1, 0, 1.0, prec, None))
    sync()
    assert rel_err(from_dev(d_out), xr - 0.37 * oracle_lib.hop(ir, gr, L, 1, False, 1.0)) <= tol
    q.check(q.lib().qcuSchurMrhs(d_out.data_ptr(), d_in.data_ptr(), d_tmp.data_ptr(), d_g.data_ptr(), 0.11,
                                 q.lattice(L), nc, m, -1.0, prec, None))
    sync()
    assert rel_err(from_dev(d_out), oracle_lib.schur(ir, gr, L, 0.11, -1.0)) <= 2 * tol
    assert q.lib().qcuGetKernelError(1) == 0


@pytest.mark.parametrize("hop_kernel", [q.HOP_SIMT, q.HOP_SIMT_CS], indirect=True, ids=["simt", "simt_cs"])
@pytest.mark.parametrize("nc,m", [(3, 4), (3, 12), (6, 8), (8, 16), (8, 32), (5, 3)])
def test_fp64_hop_kernels(oracle_lib, nc, m, hop_kernel):
    """Both SIMT work splits in FP64, with dagger and the antiperiodic boundary."""
    L = (4, 2, 4, 6)
    gauge, inp = _problem(L, nc, m, 90 + nc)
    for parity in (0, 1):
        for dagger in (False, True):
            ref = oracle_lib.hop(inp, gauge, L, parity, dagger, -1.0)
            got = _hop_gpu(inp, gauge, L, parity, dagger, -1.0, q.DOUBLE)
            assert rel_err(got, ref) <= TOL[q.DOUBLE]


@pytest.mark.parametrize("hop_kernel", [q.HOP_SIMT_CS], indirect=True, ids=["simt_cs"])
def test_colour_split_epilogues(oracle_lib, hop_kernel):
    test_xpay_and_schur_epilogues(oracle_lib)


def test_autotuner_records_a_valid_choice(tmp_path, monkeypatch):
    L = (8, 4, 4, 8)
    for prec in (q.DOUBLE, q.BF16):
        k = q.lib().qcuTuneHop(q.lattice(L), 3, 12, prec, None)
        assert k in (q.HOP_SIMT, q.HOP_SIMT_CS, q.HOP_TENSOR, q.HOP_PACKED16, q.HOP_PACKED16_PAIRS,
                     q.HOP_MMA16, q.HOP_MMA_LINK), q.last_error()
        assert q.lib().qcuGetTunedHop(3, 12, prec) == k
        if prec == q.DOUBLE:
            assert k not in (q.HOP_TENSOR, q.HOP_PACKED16, q.HOP_PACKED16_PAIRS, q.HOP_MMA16, q.HOP_MMA_LINK)
    assert q.lib().qcuTuneHop(q.lattice((7, 4, 4, 4)), 3, 12, q.DOUBLE, None) < 0


def test_xpay_and_schur_epilogues(oracle_lib):
    L, nc, m = (4, 4, 4, 4), 3, 6
    gauge, inp = _problem(L, nc, m, 50)
    x = F.to_mrhs(F.gaussian_fermions(L, nc, m, 51, parities=1)[:, 0])
    d_in, d_g, d_x = to_dev(inp), to_dev(gauge), to_dev(x)
    d_out, d_tmp = empty_dev(inp.shape), empty_dev(inp.shape)
    rc = q.lib().qcuDslashMrhsXpay(d_out.data_ptr(), d_in.data_ptr(), d_g.data_ptr(), d_x.data_ptr(), -0.37,
                                   q.lattice(L), nc, m, 0, 0, -1.0, q.DOUBLE, None)
    q.check(rc)
    sync()
    ref = x - 0.37 * oracle_lib.hop(inp, gauge, L, 0, False, -1.0)
    assert rel_err(from_dev(d_out), ref) <= 1e-13
    kappa = 0.11
    rc = q.lib().qcuSchurMrhs(d_out.data_ptr(), d_in.data_ptr(), d_tmp.data_ptr(), d_g.data_ptr(), kappa,
                              q.lattice(L), nc, m, -1.0, q.DOUBLE, None)
    q.check(rc)
    sync()
    ref = oracle_lib.schur(inp, gauge, L, kappa, -1.0)
    assert rel_err(from_dev(d_out), ref) <= 1e-13


def test_hop_rejects_bad_arguments():
    L = q.lattice((8, 8, 8, 8))
    d = empty_dev((16,))
    p = d.data_ptr()
    assert q.lib().qcuDslashMrhs(p, p, p, L, 9, 4, 0, 0, 1.0, q.DOUBLE, None) == q.ERR_UNSUPPORTED
    assert q.lib().qcuDslashMrhs(p, p, p, L, 3, 65, 0, 0, 1.0, q.DOUBLE, None) == q.ERR_INVALID
    assert q.lib().qcuDslashMrhs(p, p, p, L, 3, 4, 2, 0, 1.0, q.DOUBLE, None) == q.ERR_INVALID
    assert q.lib().qcuDslashMrhs(p, p, p, q.lattice((7, 8, 8, 8)), 3, 4, 0, 0, 1.0, q.DOUBLE, None) == q.ERR_INVALID
    assert q.lib().qcuDslashMrhs(p, p, p, L, 3, 4, 0, 0, 1.0, q.UNDEFINED, None) == q.ERR_INVALID


def _blocked_ref(a, m, nc):
    """numpy statement of the site-blocked layout: [Vh][4N][m] -> [Vh/32][4N][32][m]."""
    vh = a.shape[0]
    return a.reshape(vh // 32, 32, 4 * nc, m).transpose(0, 2, 1, 3).copy()


@pytest.mark.parametrize("prec", [q.DOUBLE, q.HALF, q.BF16])
@pytest.mark.parametrize("nc,m", [(3, 12), (2, 5), (3, 8)])
def test_site_blocked_reorder(prec, nc, m):
    """Gathered -> site-blocked is the stated permutation and comes back exactly."""
    L = (8, 8, 4, 4)
    vh = F.half_volume(L)
    rng = np.random.default_rng(5)
    a = rng.standard_normal((vh, 4, nc, m)) + 1j * rng.standard_normal((vh, 4, nc, m))
    da = to_dev(a, prec)
    db = empty_dev(a.shape, prec)
    q.check(q.lib().qcuSiteBlockMrhs(db.data_ptr(), da.data_ptr(), vh, nc, m, prec, 1, None))
    sync()
    got = from_dev(db).reshape(vh // 32, 4 * nc, 32, m)
    assert np.array_equal(got, _blocked_ref(from_dev(da).reshape(vh, 4 * nc, m), m, nc))
    back = empty_dev(a.shape, prec)
    q.check(q.lib().qcuSiteBlockMrhs(back.data_ptr(), db.data_ptr(), vh, nc, m, prec, 0, None))
    sync()
    assert np.array_equal(from_dev(back), from_dev(da))
    assert q.lib().qcuSiteBlockMrhs(db.data_ptr(), da.data_ptr(), vh - 1, nc, m, prec, 1, None) == q.ERR_INVALID
    assert q.lib().qcuSiteBlockMrhs(da.data_ptr(), da.data_ptr(), vh, nc, m, prec, 1, None) == q.ERR_INVALID


@pytest.mark.parametrize("prec", [q.HALF, q.BF16])
@pytest.mark.parametrize("m", [8, 12, 16])
@pytest.mark.parametrize("dagger", [0, 1])
def test_site_blocked_hop_matches_gathered(oracle_lib, prec, m, dagger):
    """The two-RHS packed kernel on site-blocked fields gives bit for bit the output of the
    same kernel on the gathered layout (same arithmetic, other addresses), both parities,
    antiperiodic t; and it is within the 16-bit tolerance of the oracle."""
    L, nc = (8, 4, 4, 8), 3
    vh = F.half_volume(L)
    gauge, inp = _problem(L, nc, m, 61)
    d_in, d_g = to_dev(inp, prec), to_dev(gauge, prec)
    d_bin = empty_dev(inp.shape, prec)
    q.check(q.lib().qcuSiteBlockMrhs(d_bin.data_ptr(), d_in.data_ptr(), vh, nc, m, prec, 1, None))
    q.check(q.lib().qcuSetHopKernel(q.HOP_PACKED16_PAIRS))
    try:
        for parity in (0, 1):
            d_out = empty_dev(inp.shape, prec)
            q.check(q.lib().qcuDslashMrhs(d_out.data_ptr(), d_in.data_ptr(), d_g.data_ptr(), q.lattice(L), nc, m,
                                          parity, dagger, -1.0, prec, None))
            d_bout = empty_dev(inp.shape, prec)
            q.check(q.lib().qcuDslashMrhsSiteBlocked(d_bout.data_ptr(), d_bin.data_ptr(), d_g.data_ptr(),
                                                     q.lattice(L), nc, m, parity, dagger, -1.0, prec, None))
            d_back = empty_dev(inp.shape, prec)
            q.check(q.lib().qcuSiteBlockMrhs(d_back.data_ptr(), d_bout.data_ptr(), vh, nc, m, prec, 0, None))
            sync()
            import torch
            assert torch.equal(d_back, d_out)
            ref = oracle_lib.hop(_round(inp, prec), _round(gauge, prec), L, parity, bool(dagger), -1.0)
            assert rel_err(from_dev(d_back), ref) <= TOL[prec]
    finally:
        q.lib().qcuSetHopKernel(q.HOP_AUTO)


def test_site_blocked_hop_rejects_unsupported_shapes():
    L, nc, m = (8, 4, 4, 8), 3, 12
    vh = F.half_volume(L)
    a = empty_dev((vh, 4, nc, m), q.HALF)
    g = empty_dev((4, 2, vh, nc, nc), q.HALF)
    lat = q.lattice(L)
    assert q.lib().qcuDslashMrhsSiteBlocked(a.data_ptr(), a.data_ptr(), g.data_ptr(), lat, nc, 4, 0, 0, 1.0,
                                            q.HALF, None) == q.ERR_UNSUPPORTED
    assert q.lib().qcuDslashMrhsSiteBlocked(a.data_ptr(), a.data_ptr(), g.data_ptr(), lat, nc, m, 0, 0, 1.0,
                                            q.DOUBLE, None) == q.ERR_UNSUPPORTED
    assert q.lib().qcuDslashMrhsSiteBlocked(a.data_ptr(), a.data_ptr(), g.data_ptr(), q.lattice((6, 2, 2, 2)),
                                            nc, m, 0, 0, 1.0, q.HALF, None) == q.ERR_UNSUPPORTED
