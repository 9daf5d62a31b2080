"""SU(N) generality sweep of the multi-RHS hop: every kernel that covers a shape, timed
through the C ABI (qcuDslashMrhs) with CUDA events.

  python -m qcu_mrhs_b200.sunsweep [--L 16 16 16 16] [--nc 3 4 6 8] [--m 8 16 32]
                                   [--prec f64 f32 bf16] [--reps 20]

Prints one JSON line per (N, m, precision, kernel) with the launch time, algorithmic
GB/s and GFLOP/s (hopbench's definitions), and a closing line with the fastest kernel
per (N, m, precision).  Kernels: simt (one thread per site and RHS), simt_cs (colour
split), tcgen05 (tensor cores, FP16/BF16, N <= 4), packed16 (packed 16-bit arithmetic,
FP16/BF16, N <= 4).  Inputs are random device tensors; values do not affect timing.
"""
from __future__ import annotations

import argparse
import json

from .hopbench import KERNELS, run


def applicable(kernel, nc, m, prec):
    low = prec in ("f16", "bf16")
    if kernel == "simt":
        return True
    if kernel == "simt_cs":
        return nc * m <= 256
    if kernel == "tcgen05":
        return low and 2 <= nc <= 4 and 4 * m <= 128
    if kernel == "packed16":
        return low and 2 <= nc <= 4 and m >= 2
    return False


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--L", type=int, nargs=4, default=[16, 16, 16, 16])
    ap.add_argument("--nc", type=int, nargs="+", default=[3, 4, 6, 8])
    ap.add_argument("--m", type=int, nargs="+", default=[8, 16, 32])
    ap.add_argument("--prec", nargs="+", default=["f64", "f32", "bf16"])
    ap.add_argument("--kernels", nargs="+", default=["simt", "simt_cs", "tcgen05", "packed16"])
    ap.add_argument("--reps", type=int, default=20)
    args = ap.parse_args()
    best = {}
    for nc in args.nc:
        for m in args.m:
            for prec in args.prec:
                for kname in args.kernels:
                    if not applicable(kname, nc, m, prec):
                        continue
                    r = run(tuple(args.L), nc, m, prec, args.reps, 3, kernel=KERNELS.index(kname))
                    print(json.dumps(r), flush=True)
                    key = f"N{nc}_m{m}_{prec}"
                    if key not in best or r["launch_us"] < best[key]["launch_us"]:
                        best[key] = {"kernel": kname, "launch_us": r["launch_us"], "GBps": r["GBps"],
                                     "GFLOPs": r["GFLOPs"]}
    print(json.dumps({"fastest": best}), flush=True)


if __name__ == "__main__":
    main()
