"""One configuration of the qcu.h solve, timed: the Schur BiCGStab in plain FP64 or mixed
precision, or training steps of the learned preconditioner, on seeded synthetic fields.

  python -m qcu_mrhs_b200.solvebench [--L 16 16 16 32] [--nc 3] [--m 12] [--kappa 0.124]
        [--solver plain|mixed] [--sloppy f16|bf16|f32] [--hop KIND] [--max-iter 20000]
        [--repeats 1] [--precond-steps 0]

Prints one JSON line per solve (iterations, reliable updates, solve seconds from the
library's CUDA events, FP64 true residual).  With --precond-steps K it instead runs K Adam
steps of a 4-layer, 8-channel network on random sources.  It is the driver of the kernel
profiles of the solver (one command line, small lattices) and a quick solve benchmark.
"""
from __future__ import annotations

import argparse
import ctypes
import json

PRECS = {"f16": 0, "f32": 1, "f64": 2, "bf16": 4}


def main():
    import torch

    import qcu_mrhs_b200 as q
    from qcu_mrhs_b200 import fields as F

    ap = argparse.ArgumentParser()
    ap.add_argument("--L", type=int, nargs=4, default=[16, 16, 16, 32])
    ap.add_argument("--nc", type=int, default=3)
    ap.add_argument("--m", type=int, default=12)
    ap.add_argument("--kappa", type=float, default=0.124)
    ap.add_argument("--solver", choices=["plain", "mixed"], default="plain")
    ap.add_argument("--sloppy", choices=["f16", "bf16", "f32"], default="f16")
    ap.add_argument("--hop", type=int, default=0, help="QCU_HOP_* kind of the hops (0: AUTO)")
    ap.add_argument("--max-iter", type=int, default=20000)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--repeats", type=int, default=1)
    ap.add_argument("--precond-steps", type=int, default=0)
    args = ap.parse_args()
    L, nc, m = tuple(args.L), args.nc, args.m
    lib = q.lib()
    g = torch.view_as_real(F.gauge_field_torch(L, nc, 11, kind="smooth", eps=0.3, device="cpu")).contiguous().cuda()
    if args.precond_steps:
        from qcu_mrhs_b200.precond import LearnedPreconditioner, identity_weights
        P = LearnedPreconditioner(L, nc, m, 4, 8, t_boundary=-1.0)
        P.set_weights(identity_weights(4, 8, noise=0.01, seed=1))
        P.set_gauge(g)
        vh = F.half_volume(L)
        gen = torch.Generator(device="cuda").manual_seed(5)
        b = torch.randn((2, vh, 4, nc, m, 2), device="cuda", dtype=torch.float64, generator=gen)
        for k in range(args.precond_steps):
            loss = P.train_step(b, args.kappa, 1e-3)
            print(json.dumps({"step": k, "loss": loss}), flush=True)
        P.close()
        return
    grid = q.QcuGrid((ctypes.c_int * 4)(1, 1, 1, 1))
    param = q.QcuParam((ctypes.c_int * 4)(*L))
    lib.initGridSize(ctypes.byref(grid), ctypes.byref(param), nc, m, q.DOUBLE, q.DOUBLE)
    q.check()
    lib.loadQcuGauge(g.data_ptr(), q.DOUBLE)
    lib.getDslash(0, 1.0 / (2 * args.kappa) - 4.0)
    q.check()
    o = q.default_options()
    o.solver = q.SOLVER_MIXED if args.solver == "mixed" else q.SOLVER_FUSED
    o.sloppy_precision = PRECS[args.sloppy]
    o.stop_true_residual = 1
    o.t_boundary = -1.0
    q.check(lib.qcuSetSolverOptions(ctypes.byref(o)))
    q.check(lib.qcuSetHopKernel(args.hop))
    b = F.gaussian_fermions_torch(L, nc, m, 12, device="cpu").cuda()
    ins = [torch.view_as_real(b[j]).contiguous() for j in range(m)]
    outs = [torch.empty_like(t) for t in ins]
    for r in range(args.repeats):
        for j in range(m):
            lib.pushBackFermions(outs[j].data_ptr(), ins[j].data_ptr())
        lib.qcuInvert(args.max_iter, args.tol)
        st = q.status()
        if st not in (q.SUCCESS, q.ERR_NOT_CONVERGED):   # a capped --max-iter is a valid run
            q.check(st)
        s = q.solve_stats()
        print(json.dumps({"repeat": r, "L": list(L), "nc": nc, "m": m, "solver": args.solver,
                          "sloppy": args.sloppy if args.solver == "mixed" else None,
                          "iterations": s.iterations, "reliable_updates": s.reliable_updates,
                          "solve_seconds": s.solve_seconds, "true_residual_max": max(s.true_residual[:m]),
                          "converged": st == q.SUCCESS}),
              flush=True)
    lib.qcuSetHopKernel(0)
    lib.finalizeQcu()


if __name__ == "__main__":
    main()
