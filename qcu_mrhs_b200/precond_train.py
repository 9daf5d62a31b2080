"""Train the learned gauge-covariant preconditioner on solver-generated pairs and measure
what it gains, through the library's own kernels (qcuPrecond*, qcuInvert).

  python -m qcu_mrhs_b200.precond_train [--epochs 8] [--lr 2e-3] [--out weights.npz]

Workload (defaults): 16^4 lattice, SU(3), N_rhs = 8, kappa = 0.1245, smoothed links
U = exp(i 0.3 H), antiperiodic in t.  Network: 4 parallel-transport convolution layers,
8 hidden channels, FP32 weights.  Training data: 512 pairs (b, x ~ M^-1 b), 64 per gauge
field on 8 seeded fields, x from the plain FP64 solver (tolerance 1e-10); loss
sum_j ||M P b_j - b_j||^2 / ||b_j||^2.  Test: 8 held-out seeded fields, 8 new sources each,
solved to FP64 true residual 1e-10 by
  plain      the FP64 even/odd Schur BiCGStab (the product's plain solver),
  identity   the full-system BiCGStab of QCU_SOLVER_PRECOND with P = 1 (the same method
             without the learned part),
  learned    QCU_SOLVER_PRECOND with the trained network.
Prints one JSON line per phase and a summary line.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import time

import numpy as np

L_DEFAULT = (16, 16, 16, 16)


def gathered(per_rhs):
    """list of m per-RHS full-lattice fields [2][Vh][4][N][2] -> gathered [2][Vh][4][N][m][2]"""
    import torch
    return torch.stack(per_rhs, dim=-2).contiguous()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--L", type=int, nargs=4, default=list(L_DEFAULT))
    ap.add_argument("--m", type=int, default=8)
    ap.add_argument("--kappa", type=float, default=0.1245)
    ap.add_argument("--eps", type=float, default=0.3)
    ap.add_argument("--layers", type=int, default=4)
    ap.add_argument("--channels", type=int, default=8)
    ap.add_argument("--train-fields", type=int, default=8)
    ap.add_argument("--pairs", type=int, default=512)
    ap.add_argument("--test-fields", type=int, default=8)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--out", default="")
    args = ap.parse_args()

    import torch

    import qcu_mrhs_b200 as q
    from qcu_mrhs_b200 import fields as F
    from qcu_mrhs_b200.precond import LearnedPreconditioner, identity_weights

    L, m, kappa, nc = tuple(args.L), args.m, args.kappa, 3
    lib = q.lib()
    per_field = args.pairs // args.train_fields
    batches_per_field = per_field // m

    def gauge(seed):
        g = F.gauge_field_torch(L, nc, seed, kind="smooth", eps=args.eps, device="cpu")
        return torch.view_as_real(g).contiguous().cuda()

    def sources(seed):
        b = F.gaussian_fermions_torch(L, nc, m, seed, device="cpu")
        return [torch.view_as_real(b[j]).contiguous().cuda() for j in range(m)]

    def context(dg):
        grid = q.QcuGrid((ctypes.c_int * 4)(1, 1, 1, 1))
        param = q.QcuParam((ctypes.c_int * 4)(*L))
        lib.initGridSize(ctypes.byref(grid), ctypes.byref(param), nc, m, q.DOUBLE, q.DOUBLE)
        q.check()
        lib.loadQcuGauge(dg.data_ptr(), q.DOUBLE)
        lib.getDslash(0, 1.0 / (2 * kappa) - 4.0)
        q.check()

    def solve(b, solver):
        o = q.default_options()
        o.solver = solver
        o.t_boundary = -1.0
        o.stop_true_residual = 1
        o.check_interval = 16
        q.check(lib.qcuSetSolverOptions(ctypes.byref(o)))
        x = [torch.empty_like(b[0]) for _ in range(m)]
        for j in range(m):
            lib.pushBackFermions(x[j].data_ptr(), b[j].data_ptr())
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lib.qcuInvert(20000, args.tol)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        st = q.status()
        if st != q.SUCCESS:
            raise RuntimeError(f"qcuInvert: {q.last_error()}")
        s = q.solve_stats()
        return x, {"iterations": s.iterations, "seconds": s.solve_seconds, "wall_s": wall,
                   "true_residual_max": max(s.true_residual[:m]), "fallback": s.fallback,
                   "precond_iterations": s.precond_iterations}

    # ---- training pairs from the plain solver ----
    t0 = time.perf_counter()
    data = []   # (field index, gathered b, gathered x)
    train_gauges = []
    gen_iters = []
    for f in range(args.train_fields):
        dg = gauge(5000 + f)
        train_gauges.append(dg)
        context(dg)
        for k in range(batches_per_field):
            b = sources(6000 + 100 * f + k)
            x, st = solve(b, q.SOLVER_FUSED)
            gen_iters.append(st["iterations"])
            data.append((f, gathered(b), gathered(x)))
        lib.finalizeQcu()
    print(json.dumps({"phase": "pairs", "pairs": len(data) * m, "fields": args.train_fields,
                      "plain_iterations_mean": float(np.mean(gen_iters)), "seconds": time.perf_counter() - t0}),
          flush=True)

    # ---- training ----
    P = LearnedPreconditioner(L, nc, m, args.layers, args.channels, t_boundary=-1.0)
    P.set_weights(identity_weights(args.layers, args.channels, noise=0.01, seed=1))
    rng = np.random.default_rng(0)
    t0 = time.perf_counter()
    steps = 0
    for epoch in range(args.epochs):
        lr = args.lr * (0.5 ** (epoch // max(1, args.epochs // 3)))
        losses = []
        for f in rng.permutation(args.train_fields):
            P.set_gauge(train_gauges[f])
            for idx in rng.permutation(batches_per_field):
                _, b, _ = data[f * batches_per_field + idx]
                losses.append(P.train_step(b, kappa, lr) / m)
                steps += 1
        torch.cuda.synchronize()
        print(json.dumps({"phase": "train", "epoch": epoch, "lr": lr, "loss_per_rhs": float(np.mean(losses)),
                          "seconds": time.perf_counter() - t0, "steps": steps}), flush=True)
    train_seconds = time.perf_counter() - t0
    # fit of the solver's solutions: ||P b - x|| / ||x|| on the training pairs of field 0
    P.set_gauge(train_gauges[0])
    fits = []
    for k in range(batches_per_field):
        _, b, x = data[k]
        y = torch.empty_like(b)
        P.apply(y, b)
        torch.cuda.synchronize()
        fits.append(float(torch.linalg.vector_norm(y - x) / torch.linalg.vector_norm(x)))
    del data, train_gauges
    torch.cuda.empty_cache()
    if args.out:
        np.savez(args.out, *P.get_weights())

    # ---- held-out fields ----
    ident = LearnedPreconditioner(L, nc, m, args.layers, args.channels, t_boundary=-1.0)
    ident.set_weights(identity_weights(args.layers, args.channels))
    rows = []
    for f in range(args.test_fields):
        dg = gauge(9000 + f)
        b = sources(9500 + f)
        context(dg)
        _, plain = solve(b, q.SOLVER_FUSED)
        ident.set_gauge(dg)
        ident.attach()
        _, base = solve(b, q.SOLVER_PRECOND)
        P.set_gauge(dg)
        P.attach()
        _, learned = solve(b, q.SOLVER_PRECOND)
        lib.qcuSetPreconditioner(None)
        lib.finalizeQcu()
        row = {"phase": "test", "field": f, "plain": plain, "identity": base, "learned": learned}
        rows.append(row)
        print(json.dumps(row), flush=True)

    def mean(key, sub):
        return float(np.mean([r[key][sub] for r in rows]))
    print(json.dumps({
        "phase": "summary", "lattice": list(L), "m_rhs": m, "kappa": kappa, "eps": args.eps,
        "layers": args.layers, "channels": args.channels, "pairs": args.pairs, "epochs": args.epochs,
        "train_seconds": train_seconds, "fit_rel_err_Pb_vs_x": float(np.mean(fits)),
        "iterations": {"plain_schur": mean("plain", "iterations"), "full_system_P_identity": mean("identity", "iterations"),
                       "full_system_P_learned": mean("learned", "iterations")},
        "seconds": {"plain_schur": mean("plain", "seconds"), "full_system_P_identity": mean("identity", "seconds"),
                    "full_system_P_learned": mean("learned", "seconds")},
        "iteration_gain_learned_vs_identity": mean("identity", "iterations") / mean("learned", "iterations"),
        "time_ratio_learned_vs_plain": mean("learned", "seconds") / mean("plain", "seconds"),
        "fallbacks": sum(r["learned"]["fallback"] for r in rows),
        "true_residual_max": max(max(r[k]["true_residual_max"] for k in ("plain", "identity", "learned")) for r in rows),
    }), flush=True)
    P.close()
    ident.close()


if __name__ == "__main__":
    main()
