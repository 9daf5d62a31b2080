"""qcuMrhsDotcNoAlloc: the inner product for callers that cannot allocate device memory
(their memory belongs to another allocator, or their code path forbids allocation).

It must give the same per-RHS results as qcuMrhsDotc (which allocates its scratch on
first use) on two calls in a row -- the second call reuses the fixed scratch array the
first one left behind -- allocate nothing (device free memory unchanged across its first
call in a fresh process), and reject m beyond its fixed capacity.  Collected last so a
run that stops at the first failure has run every other test already; it also passes
on its own in a fresh process.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import qcu_mrhs_b200 as q
from tests.helpers import from_dev, sync, to_dev, zeros_dev

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# the two entry points form the products and sums in FP64 at every storage precision, in
# different summation orders (their grids differ): they agree to FP64 rounding
PRECS = [(q.DOUBLE, 1e-12), (q.SINGLE, 1e-12), (q.HALF, 1e-12), (q.BF16, 1e-12)]
PREC_IDS = ["f64", "f32", "f16", "bf16"]


@pytest.mark.parametrize("prec,tol", PRECS, ids=PREC_IDS)
def test_no_alloc_dotc_matches_allocating_dotc_twice(prec, tol):
    lib = q.lib()
    rng = np.random.default_rng(123)
    for call, (n, m) in enumerate([(100003, 12), (4099, 64)]):
        a = rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))
        b = rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))
        da, db = to_dev(a, prec), to_dev(b, prec)
        want = zeros_dev((m,))
        got = zeros_dev((m,))
        q.check(lib.qcuMrhsDotcNoAlloc(got.data_ptr(), da.data_ptr(), db.data_ptr(), n, m, prec, None))
        q.check(lib.qcuMrhsDotc(want.data_ptr(), da.data_ptr(), db.data_ptr(), n, m, prec, None))
        sync()
        w, g = from_dev(want), from_dev(got)
        assert np.linalg.norm(g - w) / np.linalg.norm(w) <= tol, f"call {call}"


_CHILD = r"""
import json, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
import qcu_mrhs_b200 as q
from tests.helpers import from_dev, to_dev, zeros_dev
prec = int(sys.argv[2])
rng = np.random.default_rng(7)
n, m = 50021, 12
a = rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))
b = rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))
da, db = to_dev(a, prec), to_dev(b, prec)
got, want = zeros_dev((m,)), zeros_dev((m,))
lib = q.lib()
torch.cuda.synchronize()
free0 = torch.cuda.mem_get_info()[0]
rc = lib.qcuMrhsDotcNoAlloc(got.data_ptr(), da.data_ptr(), db.data_ptr(), n, m, prec, None)
torch.cuda.synchronize()
free1 = torch.cuda.mem_get_info()[0]
q.check(rc)
q.check(lib.qcuMrhsDotc(want.data_ptr(), da.data_ptr(), db.data_ptr(), n, m, prec, None))
torch.cuda.synchronize()
w, g = from_dev(want), from_dev(got)
print(json.dumps({"free0": free0, "free1": free1, "rel": float(np.linalg.norm(g - w) / np.linalg.norm(w))}))
"""


@pytest.mark.parametrize("prec,tol", PRECS, ids=PREC_IDS)
def test_no_alloc_dotc_first_call_allocates_nothing(prec, tol):
    """The first call of the process, before any allocating entry point: device free memory
    is the same after it as before (modules are loaded eagerly, so loading the library's
    code and its fixed scratch array happens before the measurement, not inside the call),
    and the result matches qcuMrhsDotc called afterwards."""
    env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
    res = subprocess.run([sys.executable, "-c", _CHILD, ROOT, str(prec)], capture_output=True, text=True,
                         env=env, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    d = json.loads(res.stdout.strip().splitlines()[-1])
    assert d["free1"] == d["free0"], d
    assert d["rel"] <= tol, d


def test_no_alloc_dotc_rejects_m_beyond_capacity():
    lib = q.lib()
    d = zeros_dev((65 * 4,))
    rc = lib.qcuMrhsDotcNoAlloc(d.data_ptr(), d.data_ptr(), d.data_ptr(), 4, 65, q.DOUBLE, None)
    assert rc == q.ERR_INVALID
    assert "m_rhs=65" in q.last_error()
