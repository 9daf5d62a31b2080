"""The C-ABI library loads without a GPU, exports every function that include/*.h
declares, and reports call-order errors through qcuGetLastStatus instead of aborting."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = set()
    for h in ("qcu.h", "qcu_b200.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//.*", "", text)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s*([A-Za-z_][A-Za-z0-9_]*)\s*\(",
                         text, flags=re.M):
            if m.group(1) not in ("if", "return", "sizeof"):
                names.add(m.group(1))
    return names


def test_reference_symbols_are_declared():
    names = _declared_functions()
    # reference include/qcu.h:14-29
    for f in ("initGridSize", "pushBackFermions", "loadQcuGauge", "getDslash", "start_dslash", "mat_Qcu",
              "qcuInvert", "finalizeQcu", "gauge_eo_precondition", "gauge_reverse_eo_precondition",
              "read_gauge_from_file"):
        assert f in names


def test_library_exports_every_declared_symbol(qlib):
    lib = qlib.lib()
    missing = [n for n in sorted(_declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", qlib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    assert _declared_functions() <= exported


def test_python_signatures_cover_the_headers(qlib):
    assert _declared_functions() == set(qlib._SIGNATURES)


def test_call_order_errors_are_statuses(qlib):
    lib = qlib.lib()
    lib.finalizeQcu()
    lib.start_dslash(0, 0)
    assert qlib.status() == qlib.ERR_STATE
    assert "not initialized" in qlib.last_error()
    lib.pushBackFermions(None, None)
    assert qlib.status() == qlib.ERR_STATE
    lib.getDslash(0, 0.1)
    assert qlib.status() == qlib.ERR_STATE


def test_init_rejects_bad_parameters_without_a_gpu(qlib):
    lib = qlib.lib()
    grid = qlib.QcuGrid((ctypes.c_int * 4)(1, 1, 1, 2))
    param = qlib.QcuParam((ctypes.c_int * 4)(8, 8, 8, 8))
    lib.initGridSize(ctypes.byref(grid), ctypes.byref(param), 3, 4, qlib.DOUBLE, qlib.DOUBLE)
    assert qlib.status() == qlib.ERR_UNSUPPORTED
    grid = qlib.QcuGrid((ctypes.c_int * 4)(1, 1, 1, 1))
    param = qlib.QcuParam((ctypes.c_int * 4)(7, 8, 8, 8))
    lib.initGridSize(ctypes.byref(grid), ctypes.byref(param), 3, 4, qlib.DOUBLE, qlib.DOUBLE)
    assert qlib.status() == qlib.ERR_INVALID
    param = qlib.QcuParam((ctypes.c_int * 4)(8, 8, 8, 8))
    lib.initGridSize(ctypes.byref(grid), ctypes.byref(param), 9, 4, qlib.DOUBLE, qlib.DOUBLE)
    assert qlib.status() == qlib.ERR_UNSUPPORTED
    lib.initGridSize(ctypes.byref(grid), ctypes.byref(param), 3, 0, qlib.DOUBLE, qlib.DOUBLE)
    assert qlib.status() == qlib.ERR_INVALID
    lib.initGridSize(ctypes.byref(grid), ctypes.byref(param), 3, 4, 7, qlib.DOUBLE)
    assert qlib.status() == qlib.ERR_INVALID


def test_device_entry_points_validate_before_launch(qlib):
    lib = qlib.lib()
    L = qlib.lattice((8, 8, 8, 8))
    rc = lib.qcuDslashMrhs(None, None, None, L, 3, 4, 0, 0, 1.0, qlib.DOUBLE, None)
    assert rc == qlib.ERR_INVALID
    rc = lib.qcuMrhsDotc(None, None, None, 10, 0, qlib.DOUBLE, None)
    assert rc == qlib.ERR_INVALID
    rc = lib.qcuMrhsNorm(None, None, 10, 65, qlib.DOUBLE, None)
    assert rc == qlib.ERR_INVALID


def test_batch_rejects_bad_arguments_without_a_gpu(qlib):
    lib = qlib.lib()
    assert lib.qcuInvertBatch(None, 1, None, 0) == qlib.ERR_INVALID
    arr = (qlib.QcuBatchSystem * 1)()
    assert lib.qcuInvertBatch(arr, 0, None, 0) == qlib.ERR_INVALID
    arr[0].lattice_size[:] = [4, 4, 4, 4]
    arr[0].n_color, arr[0].m_rhs, arr[0].kappa, arr[0].tol = 3, 1, 0.1, 1e-10
    assert lib.qcuInvertBatch(arr, 1, None, 0) == qlib.ERR_INVALID   # null gauge and fields
    assert "null" in qlib.last_error()


def test_precond_rejects_bad_arguments_without_a_gpu(qlib):
    import ctypes as C
    lib = qlib.lib()
    h = C.c_void_p()
    assert lib.qcuPrecondCreate(C.byref(h), qlib.lattice((7, 4, 4, 4)), 3, 4, 4, 8, 1.0) == qlib.ERR_INVALID
    assert lib.qcuPrecondCreate(C.byref(h), qlib.lattice((8, 4, 4, 4)), 5, 4, 4, 8, 1.0) == qlib.ERR_UNSUPPORTED
    assert lib.qcuPrecondCreate(C.byref(h), qlib.lattice((8, 4, 4, 4)), 3, 4, 0, 8, 1.0) == qlib.ERR_INVALID
    assert lib.qcuPrecondCreate(C.byref(h), qlib.lattice((8, 4, 4, 4)), 3, 4, 4, 8, 0.5) == qlib.ERR_INVALID
    assert not h.value
    assert lib.qcuPrecondApply(None, None, None, qlib.DOUBLE, None) == qlib.ERR_INVALID


def test_fermion_reorder_rejects_bad_arguments_without_a_gpu(qlib):
    lib = qlib.lib()
    assert lib.qcuFermionToEO(None, None, qlib.lattice((4, 4, 4, 4)), 3, qlib.DOUBLE, None) == qlib.ERR_INVALID
    assert lib.qcuFermionFromEO(1, 2, qlib.lattice((4, 4, 4, 4)), 0, qlib.DOUBLE, None) == qlib.ERR_INVALID
