"""Batched uneven solves: many independent SU(3) systems through qcuInvertBatch vs the
same systems solved one after another through the qcu.h path (qcuInvert).

  python -m qcu_mrhs_b200.batchbench [--systems 64] [--solver mixed|fp64] [--seed 4] [--out FILE]

Systems are drawn with a seeded generator: lattice from {8^4, 12^4, 16^3 x 32}, m_rhs
uniform in 1..16, kappa uniform in [0.10, 0.124], smoothed links U = exp(i eps H) with
eps uniform in [0.2, 0.5], unit complex Gaussian sources, antiperiodic in t, FP64 true
residual 1e-10.  Prints one JSON line per method: wall time of the whole batch (host
clock around the call, fields already on the device), systems/s, RHS/s, and the per-system
latency p50/p99 (batch: time from the start of the iterations to that system's
convergence, stamped on the device or observed by the host; loop: time from the start of
the loop to the end of that system's qcuInvert).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import time

import numpy as np

LATTICES = [(8, 8, 8, 8), (12, 12, 12, 12), (16, 16, 16, 32)]
TOL = 1e-10
MAX_ITER = 5000


def draw(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        L = LATTICES[int(rng.integers(len(LATTICES)))]
        m = int(rng.integers(1, 17))
        kappa = float(rng.uniform(0.10, 0.124))
        eps = float(rng.uniform(0.2, 0.5))
        out.append({"L": L, "m": m, "kappa": kappa, "eps": eps, "seed": seed * 1000 + i})
    return out


def make_device_fields(specs):
    import torch

    from qcu_mrhs_b200 import fields as F
    dev = []
    for s in specs:
        g = F.gauge_field_torch(s["L"], 3, s["seed"], kind="smooth", eps=s["eps"], device="cpu")
        b = F.gaussian_fermions_torch(s["L"], 3, s["m"], s["seed"] + 7, device="cpu")
        dg = torch.view_as_real(g).contiguous().cuda()
        db = [torch.view_as_real(b[j]).contiguous().cuda() for j in range(s["m"])]
        dx = [torch.empty_like(db[0]) for _ in range(s["m"])]
        dev.append((dg, db, dx))
    torch.cuda.synchronize()
    return dev


def options(q, solver):
    o = q.default_options()
    o.solver = q.SOLVER_MIXED if solver == "mixed" else q.SOLVER_FUSED
    o.sloppy_precision = q.HALF
    o.stop_true_residual = 1
    o.t_boundary = -1.0
    o.reliable_delta = 0.003
    o.check_interval = 16
    return o


def run_batch(q, specs, dev, opts, flags):
    import torch
    arr = (q.QcuBatchSystem * len(specs))()
    keep = []
    for i, (s, (dg, db, dx)) in enumerate(zip(specs, dev)):
        bp = q.ptr_array([t.data_ptr() for t in db])
        xp = q.ptr_array([t.data_ptr() for t in dx])
        keep += [bp, xp]
        a = arr[i]
        a.lattice_size[:] = list(s["L"])
        a.n_color, a.m_rhs, a.kappa, a.tol, a.max_iteration = 3, s["m"], s["kappa"], TOL, MAX_ITER
        a.gauge = dg.data_ptr()
        a.b = ctypes.cast(bp, ctypes.POINTER(ctypes.c_void_p))
        a.x = ctypes.cast(xp, ctypes.POINTER(ctypes.c_void_p))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rc = q.lib().qcuInvertBatch(arr, len(specs), ctypes.byref(opts), flags)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    if rc != q.SUCCESS:
        raise RuntimeError(f"qcuInvertBatch: {q.last_error()}")
    lat = [arr[i].latency_seconds for i in range(len(specs))]
    res = max(arr[i].true_residual_max for i in range(len(specs)))
    its = [arr[i].iterations for i in range(len(specs))]
    return wall, lat, res, its


def run_loop(q, specs, dev, opts):
    import torch
    lib = q.lib()
    lat, its, res = [], [], 0.0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s, (dg, db, dx) in zip(specs, dev):
        grid = q.QcuGrid((ctypes.c_int * 4)(1, 1, 1, 1))
        param = q.QcuParam((ctypes.c_int * 4)(*s["L"]))
        lib.initGridSize(ctypes.byref(grid), ctypes.byref(param), 3, s["m"], q.DOUBLE, q.DOUBLE)
        lib.loadQcuGauge(dg.data_ptr(), q.DOUBLE)
        lib.getDslash(0, 1.0 / (2 * s["kappa"]) - 4.0)
        q.check(lib.qcuSetSolverOptions(ctypes.byref(opts)))
        for j in range(s["m"]):
            lib.pushBackFermions(dx[j].data_ptr(), db[j].data_ptr())
        lib.qcuInvert(MAX_ITER, TOL)
        q.check()
        st = q.solve_stats()
        its.append(st.iterations)
        res = max(res, max(st.true_residual[:s["m"]]))
        lat.append(time.perf_counter() - t0)
    wall = time.perf_counter() - t0
    lib.finalizeQcu()
    return wall, lat, res, its


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--systems", type=int, default=64)
    ap.add_argument("--solver", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--methods", nargs="+", default=["device_loop", "host_loop", "loop"])
    ap.add_argument("--out", default=None, help="also write every line as one JSON document")
    args = ap.parse_args()
    lines = []
    import qcu_mrhs_b200 as q
    specs = draw(args.systems, args.seed)
    dev = make_device_fields(specs)
    opts = options(q, args.solver)
    n_rhs = sum(s["m"] for s in specs)
    # warm-up: kernel loading and autotuning of every shape; the batch methods keep their
    # contexts (device buffers) from this call, as a serving loop would
    run_batch(q, specs, dev, opts, q.BATCH_DEVICE_LOOP | q.BATCH_KEEP_CONTEXTS)
    for method in args.methods:
        if method == "loop":
            wall, lat, res, its = run_loop(q, specs, dev, opts)
        else:
            flags = (q.BATCH_DEVICE_LOOP if method == "device_loop" else q.BATCH_HOST_LOOP) | q.BATCH_KEEP_CONTEXTS
            wall, lat, res, its = run_batch(q, specs, dev, opts, flags)
        line = {
            "method": method, "contexts": "kept from the warm-up call" if method != "loop" else "qcu.h context per system", "solver": args.solver, "systems": len(specs), "rhs": n_rhs,
            "wall_s": wall, "systems_per_s": len(specs) / wall, "rhs_per_s": n_rhs / wall,
            "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
            "true_residual_max": res, "iterations_min_max": [min(its), max(its)],
            "lattices": {str(Lx): sum(1 for s in specs if s["L"] == Lx) for Lx in LATTICES},
        }
        lines.append(line)
        print(json.dumps(line), flush=True)
    if args.out:
        with open(args.out, "w") as f:
            json.dump({"systems": len(specs), "seed": args.seed, "solver": args.solver, "rhs": n_rhs,
                       "results": lines}, f, indent=1)


    q.lib().qcuBatchRelease()


if __name__ == "__main__":
    main()
