"""Golden vectors from the reference's own hop kernels pin the CPU oracle and the GPU path.

tests/golden/hop_*.npz were produced by tests/golden/make_golden.py, which runs the
reference's wmma hop (include/kernel/su_n_m_rhs_dslash.cuh:127-163, the kernel its
BiCGStab uses) and its SIMT hop (include/kernel/sun_mrhs_wilson_dslash_simt.cuh:203-228,
used by start_dslash / mat_Qcu), compiled from the reference's sources
(oracle/ref_build.sh) and run in FP64 on a B200.  Agreement is required to 1e-13
relative (FP64 rounding of differently ordered sums).
"""
import glob
import os

import numpy as np
import pytest

import qcu_mrhs_b200 as q
from qcu_mrhs_b200 import fields as F

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "hop_*.npz")))
TOL = 1e-13
SEED_PROJ = 3000


def _load(path):
    d = np.load(path)
    L = tuple(int(v) for v in d["L"])
    nc, m = int(d["nc"]), int(d["m"])
    if "gauge" in d:
        gauge, psi, full = d["gauge"], d["psi"], True
    else:
        gauge = F.gauge_field(L, nc, int(d["seed_gauge"]), kind=str(d["gauge_kind"]))
        psi = F.to_mrhs(F.gaussian_fermions(L, nc, m, int(d["seed_psi"]), parities=1)[:, 0])
        # the regenerated inputs must be the ones the reference kernels saw
        assert np.allclose(d["gauge_sum"], [gauge.sum(), (np.abs(gauge) ** 2).sum()], rtol=1e-12)
        assert np.allclose(d["psi_sum"], [psi.sum(), (np.abs(psi) ** 2).sum()], rtol=1e-12)
        full = False
    runs = []
    for k in d.files:
        if k.startswith("out_wmma_"):
            p, dg = k[len("out_wmma_"):].split("_")
            runs.append((int(p[1:]), int(dg[1:])))
    return d, L, nc, m, gauge, psi, full, sorted(runs)


def _project(vec, case_index):
    rng = np.random.default_rng(SEED_PROJ + case_index)
    flat = vec.reshape(-1)
    r = rng.standard_normal((64, flat.size)) + 1j * rng.standard_normal((64, flat.size))
    return r @ flat


def _case_index(path):
    from tests.golden.make_golden import CASES
    name = os.path.basename(path)[len("hop_"):-len(".npz")]
    return [c[0] for c in CASES].index(name)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_golden_fixtures_present():
    assert len(FILES) >= 6, "golden fixtures missing: run tests/golden/make_golden.py on a GPU"


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f) for f in FILES])
def test_reference_kernels_agree_with_each_other(path):
    d, L, nc, m, gauge, psi, full, runs = _load(path)
    for p, dg in runs:
        assert _rel(d[f"out_simt_p{p}_d{dg}"], d[f"out_wmma_p{p}_d{dg}"]) <= TOL


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f) for f in FILES])
def test_oracle_matches_reference_kernels(oracle_lib, path):
    d, L, nc, m, gauge, psi, full, runs = _load(path)
    ci = _case_index(path)
    for p, dg in runs:
        ours = oracle_lib.hop(psi, gauge, L, p, bool(dg), 1.0)
        if not full:
            ours = _project(ours, ci)
        for k in ("wmma", "simt"):
            assert _rel(ours, d[f"out_{k}_p{p}_d{dg}"]) <= TOL, (k, p, dg)


@pytest.mark.gpu
@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f) for f in FILES])
def test_gpu_hop_matches_reference_kernels(path):
    from tests.helpers import empty_dev, from_dev, sync, to_dev
    d, L, nc, m, gauge, psi, full, runs = _load(path)
    ci = _case_index(path)
    dg_, dp = to_dev(gauge), to_dev(psi)
    for p, dg in runs:
        out = empty_dev(psi.shape)
        q.check(q.lib().qcuDslashMrhs(out.data_ptr(), dp.data_ptr(), dg_.data_ptr(), q.lattice(L), nc, m, p, dg, 1.0,
                                      q.DOUBLE, None))
        sync()
        ours = from_dev(out)
        if not full:
            ours = _project(ours, ci)
        assert _rel(ours, d[f"out_wmma_p{p}_d{dg}"]) <= TOL
