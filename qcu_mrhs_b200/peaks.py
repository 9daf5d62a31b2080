"""Arithmetic peaks of this GPU through qcuPeakRate: FP64 and FP32 fused multiply-add on
the CUDA cores, FP64 warp MMA (m8n8k4) and FP16 / BF16 warp MMA (m16n8k16, FP32
accumulation).  These are the compute ceilings of the hop kernels (the HBM ceiling is the
copy bandwidth of MEASURED_PEAKS.json).

  python -m qcu_mrhs_b200.peaks [--iters 20000] [--repeats 5] [--out FILE]

Prints one JSON document: per kind the best and median TFLOP/s over the repeats.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import statistics

from . import PEAK_BMMA, PEAK_DFMA, PEAK_DMMA, PEAK_FFMA, PEAK_HMMA, check, lib

KINDS = {"fp64_fma": PEAK_DFMA, "fp32_fma": PEAK_FFMA, "fp64_mma_m8n8k4": PEAK_DMMA,
         "fp16_mma_m16n8k16_f32acc": PEAK_HMMA, "bf16_mma_m16n8k16_f32acc": PEAK_BMMA}


def measure(kind: int, iters: int) -> float:
    """FLOP/s of one timed launch (after a warm-up launch) on the default stream."""
    out = ctypes.c_double(0.0)
    check(lib().qcuPeakRate(kind, iters, ctypes.byref(out), None))
    return out.value


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--iters", type=int, default=20000)
    ap.add_argument("--repeats", type=int, default=5)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    res = {}
    for name, kind in KINDS.items():
        vals = [measure(kind, args.iters) / 1e12 for _ in range(args.repeats)]
        res[name] = {"tflops_best": max(vals), "tflops_median": statistics.median(vals)}
    doc = {"unit": "TFLOP/s", "iters": args.iters, "repeats": args.repeats, "peaks": res}
    print(json.dumps(doc), flush=True)
    if args.out:
        with open(args.out, "w") as f:
            json.dump(doc, f, indent=1)


if __name__ == "__main__":
    main()
