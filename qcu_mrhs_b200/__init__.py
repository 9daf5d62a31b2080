"""qcu_mrhs_b200 -- B200 (sm_100a) multi-right-hand-side SU(N) Wilson dslash and
even/odd BiCGStab behind the qcu.h C interface of qcu_mrhs.

The product is the shared library libqcu_b200.so (C ABI declared in include/qcu.h
and include/qcu_b200.h).  This module only loads it with ctypes and declares the
signatures, so Python callers (tests, the benchmark, a PyQuda-style binding) can
call it with device pointers taken from any CUDA array library.  There is no CPU
fallback: if the library is missing, `lib()` raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqcu_b200.so")

# precision codes (include/qcu_b200.h)
HALF, SINGLE, DOUBLE, UNDEFINED, BF16 = 0, 1, 2, 3, 4
PREC_BYTES = {HALF: 2, SINGLE: 4, DOUBLE: 8, BF16: 2}

# status codes
SUCCESS, ERR_INVALID, ERR_STATE, ERR_CUDA, ERR_NOT_CONVERGED, ERR_BREAKDOWN, ERR_UNSUPPORTED, ERR_ALLOC = range(8)

SOLVER_REFERENCE, SOLVER_FUSED, SOLVER_MIXED, SOLVER_PRECOND, SOLVER_CGNR = 0, 1, 2, 3, 4
(HOP_AUTO, HOP_SIMT, HOP_TENSOR, HOP_SIMT_CS, HOP_PACKED16, HOP_PACKED16_ACC16, HOP_PACKED16_STAGED,
 HOP_PACKED16_PAIRS, HOP_MMA16, HOP_MMA_LINK, HOP_MMA_LINK_DIRECT) = range(11)
PEAK_DFMA, PEAK_FFMA, PEAK_DMMA, PEAK_HMMA, PEAK_BMMA = 1, 2, 3, 4, 5
HOP_FORM_PLAIN, HOP_FORM_XPAY, HOP_FORM_SCHUR_R0, HOP_FORM_SCHUR_TS, HOP_FORM_SCHUR, HOP_FORM_RESID = range(6)
MAX_RHS = 64


class QcuParam(ctypes.Structure):
    _fields_ = [("lattice_size", ctypes.c_int * 4)]


class QcuGrid(ctypes.Structure):
    _fields_ = [("grid_size", ctypes.c_int * 4)]


class QcuSolverOptions(ctypes.Structure):
    _fields_ = [
        ("solver", ctypes.c_int),
        ("sloppy_precision", ctypes.c_int),
        ("stop_true_residual", ctypes.c_int),
        ("reliable_delta", ctypes.c_double),
        ("t_boundary", ctypes.c_double),
        ("check_interval", ctypes.c_int),
        ("freeze_converged", ctypes.c_int),
        ("max_restarts", ctypes.c_int),
        ("reliable_quorum", ctypes.c_double),
    ]


class QcuSolveStats(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int),
        ("reliable_updates", ctypes.c_int),
        ("status", ctypes.c_int),
        ("m_rhs", ctypes.c_int),
        ("true_residual", ctypes.c_double * MAX_RHS),
        ("recursive_residual", ctypes.c_double * MAX_RHS),
        ("solve_seconds", ctypes.c_double),
        ("fallback", ctypes.c_int),
        ("precond_iterations", ctypes.c_int),
    ]


class QcuBatchSystem(ctypes.Structure):
    _fields_ = [
        ("lattice_size", ctypes.c_int * 4),
        ("n_color", ctypes.c_int),
        ("m_rhs", ctypes.c_int),
        ("kappa", ctypes.c_double),
        ("tol", ctypes.c_double),
        ("max_iteration", ctypes.c_int),
        ("gauge", ctypes.c_void_p),
        ("b", ctypes.POINTER(ctypes.c_void_p)),
        ("x", ctypes.POINTER(ctypes.c_void_p)),
        ("iterations", ctypes.c_int),
        ("reliable_updates", ctypes.c_int),
        ("status", ctypes.c_int),
        ("true_residual_max", ctypes.c_double),
        ("latency_seconds", ctypes.c_double),
    ]


BATCH_DEVICE_LOOP, BATCH_HOST_LOOP, BATCH_KEEP_CONTEXTS = 0, 1, 2

_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double
_i64 = ctypes.c_int64
_ip = ctypes.POINTER(ctypes.c_int)

_SIGNATURES = {
    # qcu.h (reference signatures)
    "initGridSize": (None, [ctypes.POINTER(QcuGrid), ctypes.POINTER(QcuParam), _i, _i, _i, _i]),
    "pushBackFermions": (None, [_vp, _vp]),
    "loadQcuGauge": (None, [_vp, _i]),
    "getDslash": (None, [_i, _d]),
    "start_dslash": (None, [_i, _i]),
    "mat_Qcu": (None, [_i]),
    "qcuInvert": (None, [_i, _d]),
    "finalizeQcu": (None, []),
    "gauge_eo_precondition": (None, [_vp, _vp, _i]),
    "gauge_reverse_eo_precondition": (None, [_vp, _vp, _i]),
    "read_gauge_from_file": (None, [_vp, ctypes.c_char_p]),
    # qcu_b200.h
    "qcuGetLastStatus": (_i, []),
    "qcuGetLastError": (ctypes.c_char_p, []),
    "qcuGetDefaultSolverOptions": (None, [ctypes.POINTER(QcuSolverOptions)]),
    "qcuSetSolverOptions": (_i, [ctypes.POINTER(QcuSolverOptions)]),
    "qcuGetSolveStats": (_i, [ctypes.POINTER(QcuSolveStats)]),
    "qcuInvertBatch": (_i, [ctypes.POINTER(QcuBatchSystem), _i, ctypes.POINTER(QcuSolverOptions), _i]),
    "qcuBatchRelease": (_i, []),
    "qcuDslashMrhs": (_i, [_vp, _vp, _vp, _ip, _i, _i, _i, _i, _d, _i, _vp]),
    "qcuDslashMrhsXpay": (_i, [_vp, _vp, _vp, _vp, _d, _ip, _i, _i, _i, _i, _d, _i, _vp]),
    "qcuDslashMrhsContext": (_i, [_vp, _vp, _i, _i, _i, _vp]),
    "qcuDslashMrhsContextActive": (_i, [_vp, _vp, _i, _i, _i, _vp, _vp]),
    "qcuDslashMrhsContextForm": (_i, [_vp, _vp, _vp, _vp, _d, _i, _i, _i, _vp, _vp]),
    "qcuSchurMrhs": (_i, [_vp, _vp, _vp, _vp, _d, _ip, _i, _i, _d, _i, _vp]),
    "qcuGatherMrhs": (_i, [_vp, _i, ctypes.POINTER(_vp), _i, _i64, _i, _i, _vp]),
    "qcuScatterMrhs": (_i, [ctypes.POINTER(_vp), _i, _vp, _i, _i64, _i, _i, _vp]),
    "qcuCopyComplexVector": (_i, [_vp, _i, _vp, _i, _i64, _vp]),
    "qcuMrhsDotc": (_i, [_vp, _vp, _vp, _i64, _i, _i, _vp]),
    "qcuMrhsDotcNoAlloc": (_i, [_vp, _vp, _vp, _i64, _i, _i, _vp]),
    "qcuMrhsNorm": (_i, [_vp, _vp, _i64, _i, _i, _vp]),
    "qcuMrhsXsay": (_i, [_vp, _vp, _vp, _vp, _i64, _i, _i, _vp]),
    "qcuMrhsXpay": (_i, [_vp, _vp, _vp, _vp, _i64, _i, _i, _vp]),
    "qcuMrhsAxpby": (_i, [_vp, _vp, _vp, _vp, _vp, _i64, _i, _i, _vp]),
    "qcuMrhsAxpbypcz": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _i, _i, _vp]),
    "qcuElementwiseDiv": (_i, [_vp, _vp, _vp, _i, _vp]),
    "qcuElementwiseMul": (_i, [_vp, _vp, _vp, _i, _vp]),
    "qcuElementwiseInit": (_i, [_vp, _d, _d, _i, _vp]),
    "qcuGaugeToEO": (_i, [_vp, _vp, _ip, _i, _i, _vp]),
    "qcuGaugeFromEO": (_i, [_vp, _vp, _ip, _i, _i, _vp]),
    "qcuFermionToEO": (_i, [_vp, _vp, _ip, _i, _i, _vp]),
    "qcuFermionFromEO": (_i, [_vp, _vp, _ip, _i, _i, _vp]),
    "qcuSiteBlockMrhs": (_i, [_vp, _vp, ctypes.c_int64, _i, _i, _i, _i, _vp]),
    "qcuDslashMrhsSiteBlocked": (_i, [_vp, _vp, _vp, _ip, _i, _i, _i, _i, ctypes.c_double, _i, _vp]),
    "qcuSetHopKernel": (_i, [_i]),
    "qcuGetHopKernel": (_i, []),
    "qcuGetKernelError": (_i, [_i]),
    "qcuTuneHop": (_i, [_ip, _i, _i, _i, _vp]),
    "qcuGetTunedHop": (_i, [_i, _i, _i]),
    "qcuGetAutoHop": (_i, [_i, _i, _i]),
    "qcuDeviceSynchronize": (_i, []),
    "qcuPeakRate": (_i, [_i, _i, ctypes.POINTER(_d), _vp]),
    "qcuHopWaitSelfTest": (_i, [ctypes.c_longlong, ctypes.POINTER(_i)]),
    "qcuPrecondCreate": (_i, [ctypes.POINTER(_vp), _ip, _i, _i, _i, _i, _d]),
    "qcuPrecondDestroy": (_i, [_vp]),
    "qcuPrecondNumWeights": (_i64, [_vp]),
    "qcuPrecondSetWeights": (_i, [_vp, ctypes.POINTER(ctypes.c_float)]),
    "qcuPrecondGetWeights": (_i, [_vp, ctypes.POINTER(ctypes.c_float)]),
    "qcuPrecondSetGauge": (_i, [_vp, _vp, _i]),
    "qcuPrecondApply": (_i, [_vp, _vp, _vp, _i, _vp]),
    "qcuPrecondLossGrad": (_i, [_vp, _vp, _i, _d, ctypes.POINTER(_d), ctypes.POINTER(_d)]),
    "qcuPrecondTrainStep": (_i, [_vp, _vp, _i, _d, _d, ctypes.POINTER(_d)]),
    "qcuSetPreconditioner": (_i, [_vp]),
}

_lib = None


class QcuError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"qcu status {status}: {message}")
        self.status = status


def lib() -> ctypes.CDLL:
    """Load libqcu_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with qcu_mrhs_b200.build.build()")
        l = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def status() -> int:
    return int(lib().qcuGetLastStatus())


def last_error() -> str:
    msg = lib().qcuGetLastError()
    return msg.decode() if msg else ""


def check(rc: int | None = None) -> None:
    """Raise QcuError if `rc` (or, for void qcu.h calls, the last status) is non-zero."""
    st = status() if rc is None else int(rc)
    if st != SUCCESS:
        raise QcuError(st, last_error())


def lattice(L) -> ctypes.Array:
    return (ctypes.c_int * 4)(*[int(v) for v in L])


def default_options() -> QcuSolverOptions:
    o = QcuSolverOptions()
    lib().qcuGetDefaultSolverOptions(ctypes.byref(o))
    return o


def solve_stats() -> QcuSolveStats:
    s = QcuSolveStats()
    check(lib().qcuGetSolveStats(ctypes.byref(s)))
    return s


def ptr_array(ptrs) -> ctypes.Array:
    return (_vp * len(ptrs))(*[int(p) for p in ptrs])
