"""Micro-benchmark of the multi-RHS hop kernel through the C ABI (qcuDslashMrhs).

  python -m qcu_mrhs_b200.hopbench --L 24 24 24 48 --nc 3 --m 12 --prec bf16 --reps 20 [--context]

Prints one JSON line per precision: launch time (CUDA events on the launching
stream, after warm-up), algorithmic GB/s and GFLOP/s.  Inputs are random device
tensors (values do not affect the timing); each launch reads one parity and writes
the other, alternating, so consecutive launches do not hit a warm L2 for the
inputs of lattices larger than L2.
"""
from __future__ import annotations

import argparse
import ctypes
import json

PRECS = {"f64": 2, "f32": 1, "f16": 0, "bf16": 4}
KERNELS = ["auto", "simt", "tcgen05", "simt_cs", "packed16", "packed16_acc16", "packed16_staged", "packed16_pairs",
           "mma16", "mma_link", "mma_link_direct", "packed16_pairs_blocked"]
# the last entry is the two-RHS kernel on the site-blocked layout (qcuDslashMrhsSiteBlocked)
BLOCKED = KERNELS.index("packed16_pairs_blocked")


def hop_bytes(vh, nc, m, s):
    return vh * (8 * nc * nc * 2 * s + 2 * 4 * nc * m * 2 * s)


def hop_flops(vh, nc, m):
    return vh * m * (128 * nc * nc + 56 * nc)


def run(L, nc, m, prec_name, reps=20, warmup=3, t_sign=-1.0, kernel=0, context=False):
    import torch

    import qcu_mrhs_b200 as q
    from qcu_mrhs_b200 import fields as F
    prec = PRECS[prec_name]
    dt = {2: torch.float64, 1: torch.float32, 0: torch.float16, 4: torch.bfloat16}[prec]
    vh = F.half_volume(L)
    g = torch.randn((4, 2, vh, nc, nc, 2), device="cuda").to(dt)
    a = torch.randn((vh, 4, nc, m, 2), device="cuda").to(dt)
    b = torch.empty_like(a)
    Lc = q.lattice(L)
    st = torch.cuda.current_stream()
    sp = ctypes.c_void_p(st.cuda_stream)
    lib = q.lib()
    q.check(lib.qcuSetHopKernel(q.HOP_PACKED16_PAIRS if kernel == BLOCKED else kernel))
    if context:
        # the qcu.h context's hop (its gauge copy and, where the kernel reads them, the
        # per-site tables): what the solver runs
        grid = q.QcuGrid((ctypes.c_int * 4)(1, 1, 1, 1))
        param = q.QcuParam((ctypes.c_int * 4)(*L))
        lib.initGridSize(ctypes.byref(grid), ctypes.byref(param), nc, m, prec, prec)
        q.check()
        lib.loadQcuGauge(g.data_ptr(), prec)
        lib.getDslash(0, 1.0)
        o = q.default_options()
        o.t_boundary = t_sign
        q.check(lib.qcuSetSolverOptions(ctypes.byref(o)))

        def hop(out, inp, gp, Lc_, nc_, m_, parity, dagger, ts, pr, stream):
            return lib.qcuDslashMrhsContext(out, inp, parity, dagger, pr, stream)
    else:
        hop = lib.qcuDslashMrhsSiteBlocked if kernel == BLOCKED else lib.qcuDslashMrhs
    bufs = (a, b)
    for i in range(warmup):
        q.check(hop(bufs[(i + 1) & 1].data_ptr(), bufs[i & 1].data_ptr(), g.data_ptr(), Lc, nc, m,
                    i & 1, 0, t_sign, prec, sp))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    for i in range(reps):
        q.check(hop(bufs[(i + 1) & 1].data_ptr(), bufs[i & 1].data_ptr(), g.data_ptr(), Lc, nc, m,
                    i & 1, 0, t_sign, prec, sp))
    e1.record(st)
    torch.cuda.synchronize()
    dur = e0.elapsed_time(e1) / 1e3 / reps
    s = q.PREC_BYTES[prec]
    q.check(lib.qcuSetHopKernel(0))
    if context:
        lib.finalizeQcu()
    return {"L": list(L), "nc": nc, "m": m, "prec": prec_name, "kernel": KERNELS[kernel], "context": context,
            "launch_us": dur * 1e6,
            "GBps": hop_bytes(vh, nc, m, s) / dur / 1e9, "GFLOPs": hop_flops(vh, nc, m) / dur / 1e9,
            "algorithmic_bytes": hop_bytes(vh, nc, m, s)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--L", type=int, nargs=4, default=[24, 24, 24, 48])
    ap.add_argument("--nc", type=int, default=3)
    ap.add_argument("--m", type=int, default=12)
    ap.add_argument("--prec", nargs="+", default=["bf16", "f64"])
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--kernel", nargs="+", default=["auto"], choices=KERNELS)
    ap.add_argument("--context", action="store_true",
                    help="time qcuDslashMrhsContext (the context's hop, with its per-site tables)")
    args = ap.parse_args()
    for kname in args.kernel:
        kern = KERNELS.index(kname)
        for p in args.prec:
            print(json.dumps(run(tuple(args.L), args.nc, args.m, p, args.reps, args.warmup, kernel=kern,
                                 context=args.context)), flush=True)


if __name__ == "__main__":
    main()
