"""Multi-RHS BLAS, gather/scatter, precision casts and gauge reorder on the GPU vs the
oracle, through the C ABI.  FP64 results agree to 1e-13 relative; reductions
accumulate in FP64 for every storage precision."""
import numpy as np
import pytest

import qcu_mrhs_b200 as q
from qcu_mrhs_b200 import fields as F
from tests.helpers import empty_dev, from_dev, rel_err, sync, to_dev, zeros_dev

pytestmark = pytest.mark.gpu


def _vecs(n, m, seed, k=3):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m)) for _ in range(k)]


def _scal(m, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(m) + 1j * rng.standard_normal(m)


@pytest.mark.parametrize("m", [1, 4, 12, 64])
@pytest.mark.parametrize("n", [1, 7, 4096, 100003])
def test_dotc_and_norm_fp64(oracle_lib, m, n):
    a, b, _ = _vecs(n, m, n + m)
    da, db = to_dev(a), to_dev(b)
    res = zeros_dev((m,))
    q.check(q.lib().qcuMrhsDotc(res.data_ptr(), da.data_ptr(), db.data_ptr(), n, m, q.DOUBLE, None))
    import torch
    nrm = torch.zeros(m, dtype=torch.float64, device="cuda")
    q.check(q.lib().qcuMrhsNorm(nrm.data_ptr(), da.data_ptr(), n, m, q.DOUBLE, None))
    sync()
    assert rel_err(from_dev(res), oracle_lib.dotc(a, b, m)) <= 1e-13
    assert rel_err(nrm.cpu().numpy(), oracle_lib.norm(a, m)) <= 1e-13


def test_dotc_is_deterministic():
    a, b, _ = _vecs(300001, 12, 5)
    da, db = to_dev(a), to_dev(b)
    outs = []
    for _ in range(3):
        res = zeros_dev((12,))
        q.check(q.lib().qcuMrhsDotc(res.data_ptr(), da.data_ptr(), db.data_ptr(), 300001, 12, q.DOUBLE, None))
        sync()
        outs.append(from_dev(res))
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[1], outs[2])


@pytest.mark.parametrize("prec", [q.SINGLE, q.HALF, q.BF16])
def test_reductions_low_precision_accumulate_in_fp64(prec):
    n, m = 50000, 8
    a, b, _ = _vecs(n, m, 6)
    da, db = to_dev(a, prec), to_dev(b, prec)
    ar, br = from_dev(da), from_dev(db)
    res = zeros_dev((m,))
    q.check(q.lib().qcuMrhsDotc(res.data_ptr(), da.data_ptr(), db.data_ptr(), n, m, prec, None))
    sync()
    assert rel_err(from_dev(res), np.sum(np.conj(ar) * br, axis=0)) <= 1e-12


@pytest.mark.parametrize("m", [1, 5, 12])
def test_axpy_family_fp64(oracle_lib, m):
    n = 20011
    x, y, z = _vecs(n, m, 7 + m)
    s1, s2, s3 = _scal(m, 1), _scal(m, 2), _scal(m, 3)
    dx, dy, dz = to_dev(x), to_dev(y), to_dev(z)
    d1, d2, d3 = to_dev(s1), to_dev(s2), to_dev(s3)
    res = empty_dev((n, m))
    L = q.lib()
    q.check(L.qcuMrhsXsay(res.data_ptr(), dx.data_ptr(), d1.data_ptr(), dy.data_ptr(), n, m, q.DOUBLE, None)); sync()
    assert rel_err(from_dev(res), oracle_lib.xsay(x, s1, y, m)) <= 1e-15
    q.check(L.qcuMrhsXpay(res.data_ptr(), dx.data_ptr(), d1.data_ptr(), dy.data_ptr(), n, m, q.DOUBLE, None)); sync()
    assert rel_err(from_dev(res), oracle_lib.xpay(x, s1, y, m)) <= 1e-15
    q.check(L.qcuMrhsAxpby(res.data_ptr(), d1.data_ptr(), dx.data_ptr(), d2.data_ptr(), dy.data_ptr(), n, m,
                           q.DOUBLE, None)); sync()
    assert rel_err(from_dev(res), oracle_lib.axpby(s1, x, s2, y, m)) <= 1e-15
    q.check(L.qcuMrhsAxpbypcz(res.data_ptr(), d1.data_ptr(), dx.data_ptr(), d2.data_ptr(), dy.data_ptr(),
                              d3.data_ptr(), dz.data_ptr(), n, m, q.DOUBLE, None)); sync()
    assert rel_err(from_dev(res), oracle_lib.axpbypcz(s1, x, s2, y, s3, z, m)) <= 1e-15


def test_elementwise_scalars():
    m = 9
    x, y = _scal(m, 4), _scal(m, 5)
    dx, dy, r = to_dev(x), to_dev(y), empty_dev((m,))
    q.check(q.lib().qcuElementwiseDiv(r.data_ptr(), dx.data_ptr(), dy.data_ptr(), m, None)); sync()
    assert rel_err(from_dev(r), x / y) <= 1e-15
    q.check(q.lib().qcuElementwiseMul(r.data_ptr(), dx.data_ptr(), dy.data_ptr(), m, None)); sync()
    assert rel_err(from_dev(r), x * y) <= 1e-15
    q.check(q.lib().qcuElementwiseInit(r.data_ptr(), 0.5, -2.0, m, None)); sync()
    assert np.all(from_dev(r) == 0.5 - 2.0j)


@pytest.mark.parametrize("src_prec,dst_prec", [(q.DOUBLE, q.DOUBLE), (q.DOUBLE, q.HALF), (q.SINGLE, q.DOUBLE),
                                               (q.DOUBLE, q.BF16)])
@pytest.mark.parametrize("nc,m", [(3, 1), (3, 12), (8, 64), (5, 7)])
def test_gather_scatter_roundtrip(oracle_lib, src_prec, dst_prec, nc, m):
    L = (4, 2, 4, 2)
    vh = F.half_volume(L)
    per = F.gaussian_fermions(L, nc, m, 60 + m, parities=1)[:, 0]   # [m][vh][4][nc]
    srcs = [to_dev(per[j], src_prec) for j in range(m)]
    gathered = empty_dev((vh, 4, nc, m), dst_prec)
    q.check(q.lib().qcuGatherMrhs(gathered.data_ptr(), dst_prec, q.ptr_array([s.data_ptr() for s in srcs]),
                                  src_prec, vh, nc, m, None))
    sync()
    src_vals = np.stack([from_dev(s) for s in srcs])
    expect = F.to_mrhs(src_vals)
    got = from_dev(gathered)
    tol = {q.DOUBLE: 0, q.SINGLE: 1e-7, q.HALF: 1e-3, q.BF16: 8e-3}[dst_prec]
    assert rel_err(got, expect) <= tol
    outs = [empty_dev((vh, 4, nc), src_prec) for _ in range(m)]
    q.check(q.lib().qcuScatterMrhs(q.ptr_array([o.data_ptr() for o in outs]), src_prec, gathered.data_ptr(),
                                   dst_prec, vh, nc, m, None))
    sync()
    back = np.stack([from_dev(o) for o in outs])
    assert rel_err(back, F.from_mrhs(got)) <= (0 if src_prec == q.DOUBLE else 1e-7)


@pytest.mark.parametrize("dst", [q.SINGLE, q.HALF, q.BF16, q.DOUBLE])
def test_copy_complex_vector(dst):
    rng = np.random.default_rng(70)
    v = rng.standard_normal(1001) + 1j * rng.standard_normal(1001)
    dv = to_dev(v)
    out = empty_dev((1001,), dst)
    q.check(q.lib().qcuCopyComplexVector(out.data_ptr(), dst, dv.data_ptr(), q.DOUBLE, 1001, None))
    sync()
    got = from_dev(out)
    if dst in (q.DOUBLE, q.SINGLE):
        assert np.array_equal(got, from_dev(to_dev(v, dst)))
    else:   # round-to-nearest to 11 (FP16) or 8 (BF16) significant bits
        ulp = 2.0 ** -10 if dst == q.HALF else 2.0 ** -7
        assert np.all(np.abs(got.real - v.real) <= ulp * np.abs(v.real))
        assert np.all(np.abs(got.imag - v.imag) <= ulp * np.abs(v.imag))


@pytest.mark.parametrize("prec", [q.DOUBLE, q.SINGLE])
def test_gauge_eo_reorder(oracle_lib, prec):
    L = (4, 2, 6, 2)
    nc = 3
    V = 4 * 2 * 6 * 2
    rng = np.random.default_rng(80)
    lex = rng.standard_normal((4, V, nc, nc)) + 1j * rng.standard_normal((4, V, nc, nc))
    dl = to_dev(lex, prec)
    de = empty_dev(lex.shape, prec)
    q.check(q.lib().qcuGaugeToEO(de.data_ptr(), dl.data_ptr(), q.lattice(L), nc, prec, None))
    sync()
    assert np.array_equal(from_dev(de), oracle_lib.gauge_to_eo(from_dev(dl), L))
    back = empty_dev(lex.shape, prec)
    q.check(q.lib().qcuGaugeFromEO(back.data_ptr(), de.data_ptr(), q.lattice(L), nc, prec, None))
    sync()
    assert np.array_equal(from_dev(back), from_dev(dl))


@pytest.mark.parametrize("prec", [q.DOUBLE, q.SINGLE, q.HALF])
@pytest.mark.parametrize("L", [(4, 2, 6, 2), (2, 4, 2, 4), (6, 6, 4, 8)])
def test_fermion_eo_reorder(oracle_lib, prec, L):
    """Lexicographic <-> even/odd fermion order against the oracle; exact (a permutation)."""
    nc = 3
    V = L[0] * L[1] * L[2] * L[3]
    rng = np.random.default_rng(81)
    lex = rng.standard_normal((V, 4, nc)) + 1j * rng.standard_normal((V, 4, nc))
    dl = to_dev(lex, prec)
    de = empty_dev(lex.shape, prec)
    q.check(q.lib().qcuFermionToEO(de.data_ptr(), dl.data_ptr(), q.lattice(L), nc, prec, None))
    sync()
    ref = oracle_lib.fermion_to_eo(from_dev(dl), L)
    assert np.array_equal(from_dev(de).reshape(ref.shape), ref)
    back = empty_dev(lex.shape, prec)
    q.check(q.lib().qcuFermionFromEO(back.data_ptr(), de.data_ptr(), q.lattice(L), nc, prec, None))
    sync()
    assert np.array_equal(from_dev(back), from_dev(dl))
