"""qcuMrhsDotcNoAlloc: the inner product for callers that cannot allocate device memory
(their memory belongs to another allocator, or their code path forbids allocation).

It must give the same per-RHS results as qcuMrhsDotc (which allocates its scratch on
first use) on two calls in a row -- the second call reuses the fixed scratch array the
first one left behind -- and reject m beyond its fixed capacity.  Collected last so a
run that stops at the first failure has run every other test already; it also passes
on its own in a fresh process.
"""
import numpy as np
import pytest

import qcu_mrhs_b200 as q
from tests.helpers import from_dev, sync, to_dev, zeros_dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,tol", [(q.DOUBLE, 1e-13), (q.BF16, 1e-12)])
def test_no_alloc_dotc_matches_allocating_dotc_twice(prec, tol):
    lib = q.lib()
    rng = np.random.default_rng(123)
    for call, (n, m) in enumerate([(100003, 12), (4099, 64)]):
        a = rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))
        b = rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))
        da, db = to_dev(a, prec), to_dev(b, prec)
        want = zeros_dev((m,))
        got = zeros_dev((m,))
        q.check(lib.qcuMrhsDotc(want.data_ptr(), da.data_ptr(), db.data_ptr(), n, m, prec, None))
        q.check(lib.qcuMrhsDotcNoAlloc(got.data_ptr(), da.data_ptr(), db.data_ptr(), n, m, prec, None))
        sync()
        w, g = from_dev(want), from_dev(got)
        assert np.linalg.norm(g - w) / np.linalg.norm(w) <= tol, f"call {call}"


def test_no_alloc_dotc_rejects_m_beyond_capacity():
    lib = q.lib()
    d = zeros_dev((65 * 4,))
    rc = lib.qcuMrhsDotcNoAlloc(d.data_ptr(), d.data_ptr(), d.data_ptr(), 4, 65, q.DOUBLE, None)
    assert rc == q.ERR_INVALID
    assert "m_rhs=65" in q.last_error()
