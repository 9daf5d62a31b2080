#!/usr/bin/env python
"""Benchmark: time to solve the multi-RHS Wilson-Dirac system to an FP64 true residual
of 1e-10, mixed-precision (FP16 storage, FP32 arithmetic, FP64 reliable updates; the
BF16-storage solve is timed beside it) vs the plain FP64 BiCGStab on the same GPU and
fields, plus the dslash roofline fraction and the per-precision dslash error.

Workload: 24^3 x 48 lattice, SU(3), N_rhs = 12, kappa = 0.124, smoothed links
U = exp(i 0.3 H), unit complex Gaussian sources, antiperiodic in t.  One step = one
qcuInvert of the 12 right-hand sides.  Multi-GPU: independent replicas (one system per
GPU), max over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time-to-solve at 1e-10 FP64 residual vs plain BiCGStab; dslash % of roofline"
L = (24, 24, 24, 48)
NC, M = 3, 12
KAPPA = 0.124
EPS = 0.3
TOL = 1e-10
T_BOUNDARY = -1.0
MAX_ITER = 20000
SEED_GAUGE, SEED_SRC = 2024, 7
WORKLOAD = "24^3x48 SU(3) Wilson-Dirac, N_rhs=12, kappa=0.124, smoothed links eps=0.3, " \
           "antiperiodic t, BiCGStab to FP64 true residual 1e-10"
# Plain FP64 BiCGStab iterations this system needs (measured with this benchmark's
# plain leg on a B200); the CPU reference leg multiplies its per-iteration time by it.
PLAIN_ITERS = 44
# reliable-update rule of the mixed solves per sloppy storage: threshold delta and the
# fraction of the RHS that must meet it (a sweep of delta 0.1 .. 0.001 and quorum 0, 0.5,
# 1 on this system: FP16 is fastest at 0.003 with every RHS waiting for the others, 4
# reliable updates instead of 8; BF16 at 0.01, where the quorum changes little)
RELIABLE = {"f16": (0.003, 1.0), "bf16": (0.01, 1.0)}
CHECK_INTERVAL = 16
# DRAM bytes of one hop launch on this workload (dram__bytes.sum.per_second x
# gpu__time_duration from one ncu capture of the kernel at this size, plain epilogue);
# keyed by (storage precision, kernel)
# DRAM bytes (read + write) per launch of the plain hop on this workload, from one ncu capture
# of dram__bytes_read.sum + dram__bytes_write.sum (mean of 3 launches)
MEASURED_TRAFFIC = {("f16", "packed16_pairs"): 490.7e6, ("f16", "packed16"): 530.2e6, ("f16", "simt"): 610.6e6,
                    ("f16", "mma_link"): 651.0e6, ("bf16", "mma_link"): 647.6e6, ("f64", "simt"): 2255.7e6}
# arithmetic of each 16-bit hop kernel
DTYPE_DETAIL = {
    "mma_link_direct": "FP16 storage; spin projection in FP16 (one rounding), link products and the sum of the 8 "
                       "hops in FP32 on the tensor cores (mma.sync m16n8k16, FP32 accumulate)",
    "mma_link": "FP16 storage; spin projection in FP16 (one rounding), link products and the sum of the 8 hops "
                "in FP32 on the tensor cores (mma.sync m16n8k16, FP32 accumulate)",
    "packed16_pairs": "FP16 storage; projection and the 3-term colour sums of each link product in packed FP16, "
                      "the 8 hops summed in FP32",
    "packed16": "FP16 storage; projection and the 3-term colour sums of each link product in packed FP16, "
                "the 8 hops summed in FP32",
    "simt": "FP16 storage, FP32 arithmetic",
}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def hop_bytes(vh, nc, m, s):
    # algorithmic bytes of one half-lattice hop: 8 links + input and output spinor, once each
    return vh * (8 * nc * nc * 2 * s + 2 * 4 * nc * m * 2 * s)


def hop_flops(vh, nc, m):
    return vh * m * (128 * nc * nc + 56 * nc)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the timed region runs."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reduce_max(v, world, device):
    """Max of a per-rank value over all ranks of the initialised process group (any
    backend: NCCL on the GPUs, gloo in the CPU tests)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seeds(rank):
    """Seeds of one replica: every rank solves its own seeded system (weak scaling)."""
    return SEED_GAUGE + rank, SEED_SRC + rank


def make_fields(rank):
    """The benchmark's fields, generated on the host with torch's seeded CPU generator
    (identical for both legs): gauge [4][2][Vh][3][3] and sources [12][2][Vh][4][3]."""
    import torch
    from qcu_mrhs_b200 import fields as F
    torch.set_num_threads(os.cpu_count() or 1)
    sg, ss = replica_seeds(rank)
    gauge = F.gauge_field_torch(L, NC, sg, kind="smooth", eps=EPS, device="cpu")
    src = F.gaussian_fermions_torch(L, NC, M, ss, device="cpu")
    return gauge, src


def cpu_solve_timing(bm, gauge, plain_iters, repeats=3, n_hi=4):
    """Time-to-solve of the CPU restatement (FP64 policy-1 Schur BiCGStab, all host threads) on
    a bounded sample: `repeats` runs of setup + 1 iteration and `repeats` runs of setup +
    n_hi iterations; per-iteration time from the difference of the medians, extrapolated to
    the GPU plain solve's iteration count.  Returns value, per-iteration time, spread, sample."""
    from oracle import oracle as O

    def one(n_it):
        t0 = time.perf_counter()
        O.bicgstab(bm, gauge, L, KAPPA, n_it, TOL, t_sign=T_BOUNDARY)
        return time.perf_counter() - t0
    one(1)   # warm-up (page-in, thread pool)
    t1 = [one(1) for _ in range(repeats)]
    th = [one(n_hi) for _ in range(repeats)]
    m1, mh = statistics.median(t1), statistics.median(th)
    t_iter = max((mh - m1) / (n_hi - 1), 1e-9)
    t_setup = max(m1 - t_iter, 0.0)
    value = t_setup + t_iter * plain_iters
    spread = {"setup_plus_1_iteration_s": [min(t1), m1, max(t1)],
              f"setup_plus_{n_hi}_iterations_s": [min(th), mh, max(th)]}
    sample = (f"{repeats} x (setup + 1 iteration) and {repeats} x (setup + {n_hi} iterations) of the FP64 "
              f"policy-1 BiCGStab on the full workload ({sum(t1) + sum(th):.1f} s of CPU work); per-iteration "
              f"time from the medians, extrapolated to {plain_iters} iterations")
    return value, t_iter, spread, sample


def run_reference(args, world, rank):
    """CPU reference leg: the FP64 policy-1 Schur BiCGStab of the CPU restatement
    (the reference has no CPU implementation of its own), all host threads."""
    if rank != 0:
        return
    from oracle import oracle as O
    from qcu_mrhs_b200 import fields as F
    O.build()
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    gauge, b = make_fields(0)
    gauge = gauge.numpy()
    b = b.numpy()
    bm = np.stack([F.to_mrhs(b[:, 0]), F.to_mrhs(b[:, 1])])
    del b
    value, t_iter, spread, sample = cpu_solve_timing(bm, gauge, PLAIN_ITERS or 1,
                                                     repeats=max(3, min(args.steps, 5)))
    line = {
        "metric": METRIC, "impl": "reference", "value": value, "unit": "s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: seeded smoothed SU(3) links, unit complex Gaussian sources",
        "config": {"workload": WORKLOAD, "lattice": list(L), "n_color": NC, "m_rhs": M, "kappa": KAPPA},
        "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "port", "sample": sample,
                         "per_iteration_s": t_iter, "spread": spread},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--static-kernels", action="store_true",
                    help="use the library's static hop-kernel rule instead of the autotuner "
                         "(for profiler runs, where the tuner's timings are distorted)")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return

    import torch
    import torch.distributed as dist

    import qcu_mrhs_b200 as q
    from qcu_mrhs_b200 import fields as F

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    lib = q.lib()
    vh = F.half_volume(L)

    # ---- inputs (on the device; host copies for the end-to-end leg) ----
    gauge, src = make_fields(rank)
    d_gauge = torch.view_as_real(gauge).contiguous().cuda()
    d_src = [torch.view_as_real(src[j]).contiguous().cuda() for j in range(M)]
    d_x = [torch.empty_like(d_src[0]) for _ in range(M)]
    del gauge, src

    grid = q.QcuGrid((ctypes.c_int * 4)(1, 1, 1, 1))
    param = q.QcuParam((ctypes.c_int * 4)(*L))
    # dslash precision FP64: mat_Qcu (the independent residual check below) runs in FP64;
    # the solvers' precisions are set by the solver options
    lib.initGridSize(ctypes.byref(grid), ctypes.byref(param), NC, M, q.DOUBLE, q.DOUBLE)
    q.check()
    lib.loadQcuGauge(d_gauge.data_ptr(), q.DOUBLE)
    lib.getDslash(0, 1.0 / (2 * KAPPA) - 4.0)
    q.check()

    def set_opts(solver, sloppy=q.HALF):
        o = q.default_options()
        o.solver = solver
        o.sloppy_precision = sloppy
        o.stop_true_residual = 1
        o.t_boundary = T_BOUNDARY
        o.check_interval = CHECK_INTERVAL
        key = "bf16" if sloppy == q.BF16 else "f16"
        o.reliable_delta, o.reliable_quorum = RELIABLE[key]
        q.check(lib.qcuSetSolverOptions(ctypes.byref(o)))

    # hop kernel per (N, m, precision) picked by the autotuner before anything is timed
    tuned = {}
    names = {1: "simt", 2: "tcgen05", 3: "simt_cs", 4: "packed16", 7: "packed16_pairs", 8: "mma16", 9: "mma_link",
             10: "mma_link_direct"}
    for name, prec in (("f64", q.DOUBLE), ("f16", q.HALF), ("bf16", q.BF16)):
        if args.static_kernels:
            k = lib.qcuGetAutoHop(NC, M, prec)    # the static rule (nothing recorded)
            tuned[name] = names.get(k, str(k))
            continue
        k = lib.qcuTuneHop(q.lattice(L), NC, M, prec, None)
        if k < 0:
            raise RuntimeError(f"autotuner: {q.last_error()}")
        tuned[name] = names.get(k, str(k))
    torch.cuda.synchronize()

    def solve(srcs, outs, max_iter=MAX_ITER):
        for j in range(M):
            lib.pushBackFermions(outs[j].data_ptr(), srcs[j].data_ptr())
        lib.qcuInvert(max_iter, TOL)
        st = q.status()
        if st not in (q.SUCCESS,):
            raise RuntimeError(f"qcuInvert failed: {q.last_error()}")
        return q.solve_stats()

    d_mx = [torch.empty_like(d_src[0]) for _ in range(M)]

    def true_residual(xs):
        """max_j ||b_j - M x_j|| / ||b_j|| of the full system, recomputed in FP64 through
        mat_Qcu (independent of the solver's own statistics), outside any timed region."""
        for j in range(M):
            lib.pushBackFermions(d_mx[j].data_ptr(), xs[j].data_ptr())
        lib.mat_Qcu(0)
        q.check()
        worst = 0.0
        for j in range(M):
            worst = max(worst, float(torch.linalg.vector_norm(d_src[j] - d_mx[j]) /
                                     torch.linalg.vector_norm(d_src[j])))
        return worst

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        return reduce_max(v, world, "cuda")

    # ---- mixed precision (the product path: FP16 storage) ----
    set_opts(q.SOLVER_MIXED, q.HALF)
    for _ in range(args.warmup):
        stats = solve(d_src, d_x)
    clocks = ClockSampler(torch.cuda.current_device())
    barrier()
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    it_mixed, rel_mixed = [], []
    for _ in range(args.steps):
        stats = solve(d_src, d_x)
        it_mixed.append(stats.iterations)
        rel_mixed.append(max(stats.true_residual[:M]))
    ev1.record()
    torch.cuda.synchronize()
    t_mixed = max_over_ranks(ev0.elapsed_time(ev1) / 1e3 / args.steps)
    clk = clocks.stop()
    reliable = stats.reliable_updates
    check_mixed = true_residual(d_x)

    # ---- the same solve with BF16 storage ----
    set_opts(q.SOLVER_MIXED, q.BF16)
    solve(d_src, d_x)
    barrier()
    ev0.record()
    stats_bf = solve(d_src, d_x)
    ev1.record()
    torch.cuda.synchronize()
    t_bf16 = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
    check_bf16 = true_residual(d_x)

    # ---- plain FP64 BiCGStab (same fields, same GPU) ----
    set_opts(q.SOLVER_FUSED)
    try:
        solve(d_src, d_x, max_iter=4)
    except RuntimeError:
        pass   # warm-up of the FP64 kernels (not converged by design)
    barrier()
    ev0.record()
    stats_plain = solve(d_src, d_x)
    ev1.record()
    torch.cuda.synchronize()
    t_plain = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
    it_plain = stats_plain.iterations
    rel_plain = max(stats_plain.true_residual[:M])
    check_plain = true_residual(d_x)

    # ---- dslash roofline: the FP16 hop (dominant kernel of the solve), BF16 and FP64 beside it;
    #      dslash error of each storage precision against the FP64 hop (which matches the
    #      reference's kernels to 1e-13) on the benchmark's gauge field and a Gaussian spinor ----
    hbm, peak_kind = peaks()
    stream = torch.cuda.current_stream()
    dev_stream = ctypes.c_void_p(stream.cuda_stream)
    roof = {}
    Lc = q.lattice(L)
    gen = torch.Generator(device="cpu").manual_seed(11)
    psi64 = torch.randn((vh, 4, NC, M, 2), generator=gen, dtype=torch.float64).cuda()
    ref_out = torch.empty_like(psi64)
    # the context's own hop (qcuDslashMrhsContext): the kernel, gauge copy and per-site tables
    # the solver uses
    q.check(lib.qcuDslashMrhsContext(ref_out.data_ptr(), psi64.data_ptr(), 0, 0, q.DOUBLE, dev_stream))
    dslash_err = {}
    for name, prec, dt in (("f16", q.HALF, torch.float16), ("bf16", q.BF16, torch.bfloat16),
                           ("f32", q.SINGLE, torch.float32), ("f64", q.DOUBLE, torch.float64)):
        s_b = q.PREC_BYTES[prec]
        a = psi64.to(dt)
        out = torch.empty_like(a)
        q.check(lib.qcuDslashMrhsContext(out.data_ptr(), a.data_ptr(), 0, 0, prec, dev_stream))
        torch.cuda.synchronize()
        if prec != q.DOUBLE:
            dslash_err[name] = float(torch.linalg.vector_norm(out.double() - ref_out) /
                                     torch.linalg.vector_norm(ref_out))
        if name == "f32":
            del a, out
            continue
        for _ in range(3):
            q.check(lib.qcuDslashMrhsContext(out.data_ptr(), a.data_ptr(), 0, 0, prec, dev_stream))
        reps = 20
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for i in range(reps):
            q.check(lib.qcuDslashMrhsContext(out.data_ptr(), a.data_ptr(), i & 1, 0, prec, dev_stream))
        e1.record(stream)
        torch.cuda.synchronize()
        dur = e0.elapsed_time(e1) / 1e3 / reps
        byts = hop_bytes(vh, NC, M, s_b)
        roof[name] = {"bound": "hbm", "achieved": byts / dur / 1e9, "peak": hbm, "unit": "GB/s",
                      "frac": byts / dur / 1e9 / hbm, "traffic": MEASURED_TRAFFIC.get((name, tuned[name])),
                      "launch_us": dur * 1e6,
                      "algorithmic_bytes": byts, "gflops": hop_flops(vh, NC, M) / dur / 1e9,
                      "kernel": tuned[name], "peak_kind": f"{peak_kind} HBM copy bandwidth"}
        # the two Schur forms of every BiCGStab iteration (qcuDslashMrhsContextForm: the same
        # kernels as the solver's): out = x - kappa^2 D in with the fused sums <r0, out> or
        # <out, x>, <out, out>; their algorithmic bytes add x (and r0), each read once
        xs = torch.randn_like(psi64).to(dt)
        r0s = torch.randn_like(psi64).to(dt)
        red = torch.empty((2 * M, 2), dtype=torch.float64, device="cuda")
        spinor = vh * 4 * NC * M * 2 * s_b
        forms = {}
        for fname, form, extra in (("schur_r0", q.HOP_FORM_SCHUR_R0, 2), ("schur_ts", q.HOP_FORM_SCHUR_TS, 1)):
            def run_form(i):
                return lib.qcuDslashMrhsContextForm(out.data_ptr(), a.data_ptr(), xs.data_ptr(), r0s.data_ptr(),
                                                    KAPPA * KAPPA, form, i & 1, prec, red.data_ptr(), dev_stream)
            for i in range(3):
                q.check(run_form(i))
            torch.cuda.synchronize()
            e0.record(stream)
            for i in range(reps):
                q.check(run_form(i))
            e1.record(stream)
            torch.cuda.synchronize()
            fdur = e0.elapsed_time(e1) / 1e3 / reps
            fb = byts + extra * spinor
            forms[fname] = {"launch_us": fdur * 1e6, "algorithmic_bytes": fb, "achieved": fb / fdur / 1e9,
                            "frac": fb / fdur / 1e9 / hbm}
        roof[name]["schur_forms"] = forms
        del a, out, xs, r0s, red
    del psi64, ref_out

    # ---- end to end through the C ABI with host buffers ----
    h_gauge = torch.empty(d_gauge.shape, dtype=d_gauge.dtype, pin_memory=True)
    h_gauge.copy_(d_gauge)
    h_src = [torch.empty(d_src[0].shape, dtype=torch.float64, pin_memory=True) for _ in range(M)]
    for j in range(M):
        h_src[j].copy_(d_src[j])
    # pinned as well (empty_like does not carry pinning): the solution read-back is a DMA
    h_x = [torch.empty(d_src[0].shape, dtype=torch.float64, pin_memory=True) for _ in range(M)]
    set_opts(q.SOLVER_MIXED, q.HALF)
    barrier()
    ev0.record()
    for _ in range(args.steps):
        d_gauge.copy_(h_gauge, non_blocking=True)
        for j in range(M):
            d_src[j].copy_(h_src[j], non_blocking=True)
        torch.cuda.synchronize()
        lib.loadQcuGauge(d_gauge.data_ptr(), q.DOUBLE)
        q.check()
        solve(d_src, d_x)
        for j in range(M):
            h_x[j].copy_(d_x[j], non_blocking=True)
        torch.cuda.synchronize()
    ev1.record()
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(ev0.elapsed_time(ev1) / 1e3 / args.steps)
    h2d = h_gauge.numel() * 8 + sum(h.numel() * 8 for h in h_src)
    d2h = sum(h.numel() * 8 for h in h_x)

    # kernels launched per mixed solve: setup + 12 per graphed iteration (7 BiCGStab + 5 gated
    # reliable-update kernels) rounded up to the graph length + reconstruction/statistics
    interval = CHECK_INTERVAL
    graphed = -(-it_mixed[-1] // interval) * interval
    launches_per_solve = 4 + 9 + 12 * graphed + 1 + 4 + 4
    gpu_launches = launches_per_solve * args.steps

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(d_gauge, d_src, it_plain)

    lib.finalizeQcu()
    if rank == 0:
        line = {
            "metric": METRIC, "value": t_mixed, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_mixed * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f16",
            "dtype_detail": DTYPE_DETAIL.get(tuned["f16"], "FP16 storage, FP32 arithmetic") +
                            "; FP64 reductions, reliable updates and solution",
            "data": "synthetic: seeded smoothed SU(3) links exp(i 0.3 H), unit complex Gaussian sources",
            "config": {"workload": WORKLOAD, "lattice": list(L), "n_color": NC, "m_rhs": M, "kappa": KAPPA,
                       "tol": TOL, "l2": "inputs larger than L2 (each hop reads 478 MB in BF16, 1.9 GB in FP64)",
                       "replicas": world, "reliable_delta_quorum": RELIABLE, "check_interval": CHECK_INTERVAL,
                       "hop_kernels": tuned},
            "solves_per_s_all_ranks": world / t_mixed,
            "mixed": {"iterations": it_mixed[-1], "reliable_updates": reliable, "true_residual_max": max(rel_mixed),
                      "true_residual_check": check_mixed},
            "mixed_bf16": {"value": t_bf16, "unit": "s", "iterations": stats_bf.iterations,
                           "reliable_updates": stats_bf.reliable_updates,
                           "true_residual_max": max(stats_bf.true_residual[:M]),
                           "true_residual_check": check_bf16,
                           "speedup_vs_plain": t_plain / t_bf16},
            "true_residual_check": "max_j ||b_j - M x_j|| / ||b_j||, recomputed in FP64 with mat_Qcu from "
                                   "the returned solutions, outside the timed region",
            "dslash_rel_err_vs_fp64": dslash_err,
            "plain_fp64": {"value": t_plain, "unit": "s", "iterations": it_plain, "true_residual_max": rel_plain,
                           "true_residual_check": check_plain,
                           "speedup_mixed_vs_plain": t_plain / t_mixed},
            "roofline": roof["f16"],
            "roofline_bf16_hop": roof["bf16"],
            "roofline_fp64_hop": roof["f64"],
            "e2e": {"value": t_e2e, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "clocks": clk,
            "gpu_launches": gpu_launches,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def cpu_baseline(d_gauge, d_src, plain_iters):
    """CPU restatement (FP64 policy-1 BiCGStab), all host threads, bounded sample on the same
    fields (cpu_solve_timing)."""
    from oracle import oracle as O
    from qcu_mrhs_b200 import fields as F
    O.build()
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    g = d_gauge.cpu().numpy()
    gauge = np.ascontiguousarray(g[..., 0] + 1j * g[..., 1])
    b = np.stack([s.cpu().numpy() for s in d_src])
    b = b[..., 0] + 1j * b[..., 1]                      # [m][2][vh][4][nc]
    bm = np.stack([F.to_mrhs(b[:, 0]), F.to_mrhs(b[:, 1])])
    del b, g
    value, t_iter, spread, sample = cpu_solve_timing(bm, gauge, plain_iters)
    return {"value": value, "unit": "s", "cores": threads, "kind": "port", "sample": sample,
            "per_iteration_s": t_iter, "spread": spread}


if __name__ == "__main__":
    main()
