"""qcuPeakRate: the arithmetic ceilings the hop kernels are compared with.  Each kind
returns a positive FLOP rate, the warp MMAs beat the CUDA-core FMAs of their precision
class, and FP32 FMA beats FP64 FMA (B200: about 34, 72, 37 and 556 TFLOP/s)."""
import ctypes

import pytest

import qcu_mrhs_b200 as q

pytestmark = pytest.mark.gpu


def _rate(kind, iters=2000):
    out = ctypes.c_double(0.0)
    q.check(q.lib().qcuPeakRate(kind, iters, ctypes.byref(out), None))
    return out.value


def test_peak_rates_are_ordered():
    r = {k: _rate(k) for k in (q.PEAK_DFMA, q.PEAK_FFMA, q.PEAK_DMMA, q.PEAK_HMMA, q.PEAK_BMMA)}
    assert all(v > 1e12 for v in r.values()), r
    assert r[q.PEAK_FFMA] > 1.5 * r[q.PEAK_DFMA], r
    assert r[q.PEAK_HMMA] > 4 * r[q.PEAK_FFMA] and r[q.PEAK_BMMA] > 4 * r[q.PEAK_FFMA], r


def test_peak_rate_rejects_bad_arguments():
    out = ctypes.c_double(0.0)
    assert q.lib().qcuPeakRate(99, 10, ctypes.byref(out), None) == q.ERR_INVALID
    assert q.lib().qcuPeakRate(q.PEAK_DFMA, 0, ctypes.byref(out), None) == q.ERR_INVALID
    assert q.lib().qcuPeakRate(q.PEAK_DFMA, 10, None, None) == q.ERR_INVALID
