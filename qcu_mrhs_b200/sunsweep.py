"""SU(N) generality sweep of the multi-RHS hop: every kernel that covers a shape, timed
through the C ABI (qcuDslashMrhs) with CUDA events.

  python -m qcu_mrhs_b200.sunsweep [--L 16 16 16 16] [--nc 2 3 4 5 6 7 8] [--m 8 16 32]
                                   [--prec f64 f32 f16 bf16] [--reps 20] [--out FILE]

Prints one JSON line per (N, m, precision, kernel) with the launch time, algorithmic
GB/s and GFLOP/s (hopbench's definitions) and the fraction of the HBM copy bandwidth
(MEASURED_PEAKS.json at the repository root, else 6650 GB/s), and a closing line with the
fastest kernel per (N, m, precision) and, per (N, m), the speed-up of the fastest 16-bit
kernel over the fastest FP32 one.  --out also writes all of it as one JSON document.
Kernels: simt (one thread per site and RHS), simt_cs (colour split), tcgen05 (tensor
cores, FP16/BF16, N <= 4), packed16 (packed 16-bit arithmetic, FP16/BF16, N <= 4),
mma_link (warp MMA with the links as the A operand, FP16/BF16, 2 <= N <= 8).  Every hop
is the qcu.h context's (qcuDslashMrhsContext: what the solver runs, with the per-site
tables where the kernel reads them).  Inputs are random device tensors; values do not
affect timing.

Tensor-pipe utilisation: run the sweep once more under ncu with only the tensor-core
kernel and one timed launch per shape,

  ncu --metrics sm__pipe_tensor_cycles_active.avg.pct_of_peak_sustained_active \
      --clock-control none -k regex:hop_mmal --csv --log-file T.csv \
      python -m qcu_mrhs_b200.sunsweep --kernels mma_link --reps 1 [same shape options]

then `python -m qcu_mrhs_b200.sunsweep --merge-ncu T.csv --into FILE [same shape options]`
adds `tensor_pipe_pct` (the last captured launch of each shape) to the mma_link rows of
FILE, and 0 to the SIMT rows (no tensor-core instructions).
"""
from __future__ import annotations

import argparse
import json
import os

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
    if kernel == "mma_link":
        return low and 2 <= nc <= 8
    if kernel == "mma_link_direct":   # differs from mma_link only where that one stages
        return low and 2 <= nc <= 4 and m <= 16 and m % 4 == 0
    return False


def merge_ncu(csv_path, json_path, shapes, warmup=3, reps=1):
    """Attach the tensor-pipe utilisation of an ncu capture of `--kernels mma_link --reps
    reps` to the rows of the sweep document json_path.  `shapes` lists the (N, m, prec) of
    the captured sweep in order; each took warmup + reps launches."""
    import csv
    metric = "sm__pipe_tensor_cycles_active.avg.pct_of_peak_sustained_active"
    vals = []
    with open(csv_path) as f:
        lines = [ln for ln in f if ln.startswith('"')]
    for row in csv.DictReader(lines):
        if row.get("Metric Name") == metric:
            vals.append(float(row["Metric Value"].replace(",", "")))
    per = warmup + reps
    if len(vals) != per * len(shapes):
        raise SystemExit(f"{len(vals)} captured launches for {len(shapes)} shapes x {per}")
    pipe = {shape: vals[(i + 1) * per - 1] for i, shape in enumerate(shapes)}
    with open(json_path) as f:
        doc = json.load(f)
    for r in doc["rows"]:
        key = (r["nc"], r["m"], r["prec"])
        if r["kernel"] == "mma_link" and key in pipe:
            r["tensor_pipe_pct"] = pipe[key]
        elif r["kernel"] in ("simt", "simt_cs"):
            r["tensor_pipe_pct"] = 0.0
    for key, b in doc["fastest"].items():
        nc, m, prec = int(key.split("_")[0][1:]), int(key.split("_")[1][1:]), key.split("_")[2]
        if b["kernel"] == "mma_link" and (nc, m, prec) in pipe:
            b["tensor_pipe_pct"] = pipe[(nc, m, prec)]
        elif b["kernel"] in ("simt", "simt_cs"):
            b["tensor_pipe_pct"] = 0.0
    doc["tensor_pipe_source"] = "ncu sm__pipe_tensor_cycles_active.avg.pct_of_peak_sustained_active, one launch per shape"
    with open(json_path, "w") as f:
        json.dump(doc, f, indent=1)


def hbm_peak():
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--L", type=int, nargs=4, default=[16, 16, 16, 16])
    ap.add_argument("--nc", type=int, nargs="+", default=[2, 3, 4, 5, 6, 7, 8])
    ap.add_argument("--m", type=int, nargs="+", default=[8, 16, 32])
    ap.add_argument("--prec", nargs="+", default=["f64", "f32", "f16", "bf16"])
    ap.add_argument("--kernels", nargs="+", default=["simt", "simt_cs", "tcgen05", "packed16", "mma_link",
                                                      "mma_link_direct"])
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--out", default=None, help="also write every line as one JSON document")
    ap.add_argument("--merge-ncu", default=None, help="ncu CSV of a --kernels mma_link --reps 1 sweep")
    ap.add_argument("--into", default=None, help="sweep document to add tensor_pipe_pct to")
    args = ap.parse_args()
    if args.merge_ncu:
        shapes = [(nc, m, prec) for nc in args.nc for m in args.m for prec in args.prec
                  if applicable("mma_link", nc, m, prec)]
        merge_ncu(args.merge_ncu, args.into, shapes)
        return
    peak, peak_kind = hbm_peak()
    best = {}
    rows = []
    for nc in args.nc:
        for m in args.m:
            for prec in args.prec:
                for kname in args.kernels:
                    if not applicable(kname, nc, m, prec):
                        continue
                    r = run(tuple(args.L), nc, m, prec, args.reps, 3, kernel=KERNELS.index(kname), context=True)
                    r["hbm_frac"] = r["GBps"] / peak
                    rows.append(r)
                    print(json.dumps(r), flush=True)
                    key = f"N{nc}_m{m}_{prec}"
                    if key not in best or r["launch_us"] < best[key]["launch_us"]:
                        best[key] = {"kernel": kname, "launch_us": r["launch_us"], "GBps": r["GBps"],
                                     "GFLOPs": r["GFLOPs"], "hbm_frac": r["hbm_frac"]}
    # per (N, m): fastest 16-bit kernel against the fastest FP32 one (time ratio)
    low_vs_f32 = {}
    for nc in args.nc:
        for m in args.m:
            f32 = best.get(f"N{nc}_m{m}_f32")
            for lp in ("f16", "bf16"):
                b = best.get(f"N{nc}_m{m}_{lp}")
                if f32 and b:
                    low_vs_f32[f"N{nc}_m{m}_{lp}"] = f32["launch_us"] / b["launch_us"]
    summary = {"fastest": best, "speedup_vs_f32": low_vs_f32, "hbm_peak_gbs": peak, "hbm_peak_kind": peak_kind}
    print(json.dumps(summary), flush=True)
    if args.out:
        with open(args.out, "w") as f:
            json.dump({"L": args.L, "reps": args.reps, "rows": rows, **summary}, f, indent=1)


if __name__ == "__main__":
    main()
