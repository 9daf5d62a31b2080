// solver.cu -- even/odd Schur BiCGStab on the gathered multi-RHS fields.
//
// Schur system (reference src/solver/bicgstab.cu:141-189, bicgstab_solve.cu:27-70, 688-740):
//   b'_o = b_o + kappa D_oe b_e ;  A x_o = (1 - kappa^2 D_oe D_eo) x_o = b'_o ;
//   x_e  = b_e + kappa D_eo x_o.
//
// solve_fused: the reference's policy-1 iteration (per-RHS alpha, omega, beta; x0 = 0;
//   r0 = r = p = b'; stop when every RHS has ||r_j|| <= tol ||b'_j||, or the full-system
//   norm with stop_true_residual) as 8 kernels per iteration (4 hops with fused
//   epilogues and reductions, 4 fused vector updates), with all scalars in device memory
//   and `check_interval` iterations captured in one CUDA graph between host checks.
// solve_mixed: the same iteration on sloppy-precision vectors and gauge (FP32, FP16 or
//   BF16 storage, FP32 arithmetic, FP64 reductions), solution increments accumulated in
//   FP32, and reliable updates in FP64: x += e, r = b' - A x recomputed in FP64 whenever
//   the sloppy residual has fallen by `reliable_delta` or claims convergence; the solve
//   stops only on the FP64 true residual.
#include <cmath>
#include <cstring>
#include <functional>

#include "blas.h"
#include "context.h"
#include "dslash.h"

namespace qcub {

namespace {

struct Hop {
    Context& c;
    int prec;
    const void* gauge;
    int launch(void* out, const void* in, int parity, int epi, const void* x = nullptr,
               const void* r0 = nullptr, double a = 0.0, int fin = FIN_NONE, BicgScalars* sc = nullptr,
               double2* result = nullptr, const int* done = nullptr, const int* gate = nullptr) {
        HopParams p{};
        p.out = out;
        p.in = in;
        p.gauge = gauge;
        p.x = x;
        p.r0 = r0;
        p.g = c.g;
        p.m = c.m;
        p.parity = parity;
        p.t_sign = c.opts.t_boundary;
        p.a = a;
        p.red = RedArgs{c.ws.partials, c.ws.counter, result ? result : c.ws.result, sc, nullptr, fin};
        p.done = done;
        p.gate = gate;
        return hop_launch(p, c.nc, prec, false, epi, c.stream);
    }
};

int capture(Context& c, int count, const std::function<int()>& body, cudaGraphExec_t* exec) {
    cudaGraph_t graph = nullptr;
    QCUB_CUDA_CHECK(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
    int rc = QCU_SUCCESS;
    for (int i = 0; i < count && rc == QCU_SUCCESS; ++i) rc = body();
    const cudaError_t e = cudaStreamEndCapture(c.stream, &graph);
    if (rc != QCU_SUCCESS) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return set_error(QCU_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    const cudaError_t ei = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) return set_error(QCU_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ei));
    return QCU_SUCCESS;
}

// Run the captured iteration block until the device sets `done`.
int run_graph(Context& c, cudaGraphExec_t exec, BicgScalars* dsc) {
    for (;;) {
        QCUB_CUDA_CHECK(cudaGraphLaunch(exec, c.stream));
        QCUB_CUDA_CHECK(cudaMemcpyAsync(c.host_sc, dsc, sizeof(BicgScalars), cudaMemcpyDeviceToHost, c.stream));
        QCUB_CUDA_CHECK(cudaStreamSynchronize(c.stream));
        if (c.host_sc->done) return QCU_SUCCESS;
    }
}

__global__ void set_bfull_kernel(BicgScalars* sc, const double2* ne, const double2* no, int m,
                                 int use_for_stop) {
    const int j = threadIdx.x;
    if (j >= m) return;
    const double b2 = ne[j].x + no[j].x;
    sc->bfull2[j] = b2;
    if (use_for_stop) sc->bnorm2[j] = b2;
}

int prepare_scalars(Context& c, BicgScalars* dsc, int max_iter, double tol, int mixed) {
    BicgScalars& h = *c.host_sc;
    std::memset(&h, 0, sizeof(BicgScalars));
    h.m = c.m;
    h.tol2 = tol * tol;
    h.freeze = c.opts.freeze_converged ? 1 : 0;
    h.max_iter = max_iter;
    h.mixed = mixed;
    h.delta = c.opts.reliable_delta > 0 ? c.opts.reliable_delta : 0.1;
    h.len_per_rhs = (double)c.half_len();
    for (int j = 0; j < c.m; ++j) {
        h.active[j] = 1;
        h.scale[j] = 1.0;
        h.ratio[j] = 1.0;
        h.maxr[j] = 1.0;
    }
    if (max_iter <= 0) {
        h.done = 1;
        h.status = 3;
    }
    QCUB_CUDA_CHECK(cudaMemcpyAsync(dsc, &h, sizeof(BicgScalars), cudaMemcpyHostToDevice, c.stream));
    QCUB_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    return QCU_SUCCESS;
}

// ||b - M x|| / ||b|| per RHS on the full system, FP64 (or the solve precision).
int true_residual(Context& c, int prec, const void* gauge, const void* x, const void* b, void* tmp,
                  double2* slots, double* rel) {
    const size_t hb = c.half_bytes(prec);
    const char* xe = static_cast<const char*>(x);
    const char* be = static_cast<const char*>(b);
    Hop hop{c, prec, gauge};
    // r_e = b_e - (x_e - kappa D_eo x_o) ; r_o = b_o - (x_o - kappa D_oe x_e)
    int rc = hop.launch(tmp, xe + hb, 0, EPI_RESID, xe, be, c.kappa, FIN_NONE, nullptr, slots + 0 * kMaxRhs);
    if (rc) return rc;
    rc = hop.launch(tmp, xe, 1, EPI_RESID, xe + hb, be + hb, c.kappa, FIN_NONE, nullptr, slots + 1 * kMaxRhs);
    if (rc) return rc;
    rc = mrhs_dotc(slots + 2 * kMaxRhs, be, be, c.half_len(), c.m, prec, c.ws, c.stream);
    if (rc) return rc;
    rc = mrhs_dotc(slots + 3 * kMaxRhs, be + hb, be + hb, c.half_len(), c.m, prec, c.ws, c.stream);
    if (rc) return rc;
    double2 h[4 * kMaxRhs];
    QCUB_CUDA_CHECK(cudaMemcpyAsync(h, slots, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
    QCUB_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    for (int j = 0; j < c.m; ++j) {
        const double r2 = h[j].x + h[kMaxRhs + j].x;
        const double b2 = h[2 * kMaxRhs + j].x + h[3 * kMaxRhs + j].x;
        rel[j] = b2 > 0 ? std::sqrt(r2 / b2) : std::sqrt(r2);
    }
    return QCU_SUCCESS;
}

int finish_stats(Context& c, int prec, const void* gauge, const void* x, const void* b, void* tmp,
                 double2* slots) {
    QcuSolveStats& st = c.stats;
    st.m_rhs = c.m;
    st.iterations = c.host_sc->iter;
    st.reliable_updates = c.host_sc->reliable;
    st.status = c.host_sc->status == 1 ? QCU_SUCCESS
                : (c.host_sc->status == 2 ? QCU_ERR_BREAKDOWN : QCU_ERR_NOT_CONVERGED);
    for (int j = 0; j < c.m; ++j) {
        const double b2 = c.host_sc->bnorm2[j];
        st.recursive_residual[j] = b2 > 0 ? std::sqrt(c.host_sc->rnorm2[j] / b2) : 0.0;
    }
    return true_residual(c, prec, gauge, x, b, tmp, slots, st.true_residual);
}

}  // namespace

int solve_fused(Context& c, void* x, const void* b, int max_iter, double tol) {
    const int P = c.in_prec;
    if (P != QCU_PRECISION_DOUBLE && P != QCU_PRECISION_SINGLE)
        return set_error(QCU_ERR_UNSUPPORTED, "the solve precision must be double or single");
    const void* gauge = nullptr;
    int rc = c.gauge_in(P, &gauge);
    if (rc) return rc;
    const size_t hb = c.half_bytes(P);
    for (int i = 0; i < 8; ++i)
        if ((rc = c.sv[i].ensure(hb))) return rc;
    if ((rc = c.sv[15].ensure(sizeof(double2) * 8 * kMaxRhs))) return rc;
    void* bp = c.sv[0].ptr; void* r0 = c.sv[1].ptr; void* r = c.sv[2].ptr; void* p = c.sv[3].ptr;
    void* v = c.sv[4].ptr; void* s = c.sv[5].ptr; void* t = c.sv[6].ptr; void* tmp = c.sv[7].ptr;
    double2* slots = static_cast<double2*>(c.sv[15].ptr);
    BicgScalars* dsc = static_cast<BicgScalars*>(c.scalars.ptr);
    const char* be = static_cast<const char*>(b);
    const void* bo = be + hb;
    char* xe = static_cast<char*>(x);
    void* xo = xe + hb;
    const int64_t len = c.half_len();
    const double k2 = c.kappa * c.kappa;
    Hop hop{c, P, gauge};

    QCUB_CUDA_CHECK(cudaEventRecord(c.ev0, c.stream));
    if ((rc = prepare_scalars(c, dsc, max_iter, tol, 0))) return rc;
    // b' = b_o + kappa D_oe b_e
    if ((rc = hop.launch(bp, be, 1, EPI_XPAY, bo, nullptr, c.kappa))) return rc;
    BicgStepArgs a;
    a.src = bp; a.r0 = r0; a.r = r; a.p = p; a.v = v; a.s = s; a.t = t; a.x = xo;
    a.sc = dsc; a.ws = c.ws; a.len = len; a.m = c.m;
    if ((rc = bicg_step(STEP_INIT, P, P, a, c.stream))) return rc;
    // full-system norms of b (stopping reference with stop_true_residual)
    if ((rc = mrhs_dotc(slots + 4 * kMaxRhs, be, be, len, c.m, P, c.ws, c.stream))) return rc;
    if ((rc = mrhs_dotc(slots + 5 * kMaxRhs, bo, bo, len, c.m, P, c.ws, c.stream))) return rc;
    set_bfull_kernel<<<1, 64, 0, c.stream>>>(dsc, slots + 4 * kMaxRhs, slots + 5 * kMaxRhs, c.m,
                                             c.opts.stop_true_residual ? 1 : 0);
    QCUB_CHECK_LAUNCH();

    const int* done = &dsc->done;
    auto iteration = [&]() -> int {
        int e;
        if ((e = hop.launch(tmp, p, 0, EPI_PLAIN, nullptr, nullptr, 0.0, FIN_NONE, nullptr, nullptr, done))) return e;
        if ((e = hop.launch(v, tmp, 1, EPI_SCHUR_R0, p, r0, k2, FIN_ALPHA, dsc, dsc->red[0], done))) return e;
        if ((e = bicg_step(STEP_S, P, P, a, c.stream))) return e;
        if ((e = hop.launch(tmp, s, 0, EPI_PLAIN, nullptr, nullptr, 0.0, FIN_NONE, nullptr, nullptr, done))) return e;
        if ((e = hop.launch(t, tmp, 1, EPI_SCHUR_TS, s, nullptr, k2, FIN_OMEGA, dsc, dsc->red[0], done))) return e;
        if ((e = bicg_step(STEP_XR, P, P, a, c.stream))) return e;
        return bicg_step(STEP_P, P, P, a, c.stream);
    };
    const int interval = c.opts.check_interval > 0 ? c.opts.check_interval : 8;
    cudaGraphExec_t exec = nullptr;
    if ((rc = capture(c, interval, iteration, &exec))) return rc;
    rc = run_graph(c, exec, dsc);
    cudaGraphExecDestroy(exec);
    if (rc) return rc;
    // x_e = b_e + kappa D_eo x_o
    if ((rc = hop.launch(xe, xo, 0, EPI_XPAY, be, nullptr, c.kappa))) return rc;
    QCUB_CUDA_CHECK(cudaEventRecord(c.ev1, c.stream));
    if ((rc = finish_stats(c, P, gauge, x, b, tmp, slots))) return rc;
    float ms = 0.f;
    QCUB_CUDA_CHECK(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
    c.stats.solve_seconds = ms * 1e-3;
    if (c.stats.status != QCU_SUCCESS)
        return set_error(c.stats.status, "BiCGStab stopped after %d iterations (%s)", c.stats.iterations,
                         c.stats.status == QCU_ERR_BREAKDOWN ? "breakdown" : "max_iteration reached");
    return QCU_SUCCESS;
}

int solve_mixed(Context& c, void* x, const void* b, int max_iter, double tol) {
    if (c.in_prec != QCU_PRECISION_DOUBLE)
        return set_error(QCU_ERR_UNSUPPORTED, "mixed precision needs double-precision fields");
    const int S = c.opts.sloppy_precision;
    if (S != QCU_PRECISION_SINGLE && S != QCU_PRECISION_HALF && S != QCU_PRECISION_BF16)
        return set_error(QCU_ERR_INVALID, "sloppy precision %d (single, half or bf16)", S);
    const int D = QCU_PRECISION_DOUBLE;
    const void* g64 = nullptr;
    const void* gs = nullptr;
    int rc;
    if ((rc = c.gauge_in(D, &g64))) return rc;
    if ((rc = c.gauge_in(S, &gs))) return rc;
    const size_t hb = c.half_bytes(D);
    const size_t hs = c.half_bytes(S);
    const size_t he = c.half_bytes(QCU_PRECISION_SINGLE);
    for (int i = 0; i < 3; ++i)
        if ((rc = c.sv[i].ensure(hb))) return rc;
    for (int i = 3; i < 10; ++i)
        if ((rc = c.sv[i].ensure(hs))) return rc;
    if ((rc = c.sv[10].ensure(he))) return rc;
    if ((rc = c.sv[15].ensure(sizeof(double2) * 8 * kMaxRhs))) return rc;
    void* bp = c.sv[0].ptr; void* r64 = c.sv[1].ptr; void* tmp64 = c.sv[2].ptr;
    void* r0s = c.sv[3].ptr; void* rs = c.sv[4].ptr; void* ps = c.sv[5].ptr; void* vs = c.sv[6].ptr;
    void* ss = c.sv[7].ptr; void* ts = c.sv[8].ptr; void* tmps = c.sv[9].ptr; void* e = c.sv[10].ptr;
    double2* slots = static_cast<double2*>(c.sv[15].ptr);
    BicgScalars* dsc = static_cast<BicgScalars*>(c.scalars.ptr);
    const char* be = static_cast<const char*>(b);
    const void* bo = be + hb;
    char* xe = static_cast<char*>(x);
    void* xo = xe + hb;
    const int64_t len = c.half_len();
    const double k2 = c.kappa * c.kappa;
    Hop h64{c, D, g64};
    Hop hs_{c, S, gs};

    QCUB_CUDA_CHECK(cudaEventRecord(c.ev0, c.stream));
    if ((rc = prepare_scalars(c, dsc, max_iter, tol, 1))) return rc;
    // b' = b_o + kappa D_oe b_e (FP64); ||b||^2 of the full system
    if ((rc = h64.launch(bp, be, 1, EPI_XPAY, bo, nullptr, c.kappa))) return rc;
    if ((rc = mrhs_dotc(slots + 4 * kMaxRhs, be, be, len, c.m, D, c.ws, c.stream))) return rc;
    if ((rc = mrhs_dotc(slots + 5 * kMaxRhs, bo, bo, len, c.m, D, c.ws, c.stream))) return rc;
    set_bfull_kernel<<<1, 64, 0, c.stream>>>(dsc, slots + 4 * kMaxRhs, slots + 5 * kMaxRhs, c.m, 1);
    QCUB_CHECK_LAUNCH();
    // x_o = 0, r64 = b', e = 0, rtrue2 = ||b'||^2
    QCUB_CUDA_CHECK(cudaMemsetAsync(xo, 0, hb, c.stream));
    QCUB_CUDA_CHECK(cudaMemsetAsync(e, 0, he, c.stream));
    QCUB_CUDA_CHECK(cudaMemcpyAsync(r64, bp, hb, cudaMemcpyDeviceToDevice, c.stream));
    if ((rc = mrhs_norm(nullptr, r64, len, c.m, D, c.ws, c.stream, FIN_RNORM, dsc))) return rc;
    if ((rc = mp_update(dsc, c.m, 1, c.stream))) return rc;
    if ((rc = mp_load(S, rs, ps, r0s, r64, dsc, len, c.m, 1, c.ws, c.stream))) return rc;

    BicgStepArgs a;
    a.r0 = r0s; a.r = rs; a.p = ps; a.v = vs; a.s = ss; a.t = ts; a.x = e;
    a.sc = dsc; a.ws = c.ws; a.len = len; a.m = c.m;
    const int* done = &dsc->done;
    const int* gate = &dsc->gate;
    const int XP = QCU_PRECISION_SINGLE;
    auto iteration = [&]() -> int {
        int q;
        // sloppy BiCGStab iteration
        if ((q = hs_.launch(tmps, ps, 0, EPI_PLAIN, nullptr, nullptr, 0.0, FIN_NONE, nullptr, nullptr, done))) return q;
        if ((q = hs_.launch(vs, tmps, 1, EPI_SCHUR_R0, ps, r0s, k2, FIN_ALPHA, dsc, dsc->red[0], done))) return q;
        if ((q = bicg_step(STEP_S, S, XP, a, c.stream))) return q;
        if ((q = hs_.launch(tmps, ss, 0, EPI_PLAIN, nullptr, nullptr, 0.0, FIN_NONE, nullptr, nullptr, done))) return q;
        if ((q = hs_.launch(ts, tmps, 1, EPI_SCHUR_TS, ss, nullptr, k2, FIN_OMEGA, dsc, dsc->red[0], done))) return q;
        if ((q = bicg_step(STEP_XR, S, XP, a, c.stream))) return q;
        if ((q = bicg_step(STEP_P, S, XP, a, c.stream))) return q;
        // reliable update (every kernel returns at once unless one is pending)
        if ((q = mp_accum(xo, e, dsc, len, c.m, c.stream))) return q;
        if ((q = h64.launch(tmp64, xo, 0, EPI_PLAIN, nullptr, nullptr, 0.0, FIN_NONE, nullptr, nullptr, done, gate))) return q;
        if ((q = h64.launch(r64, tmp64, 1, EPI_RESID, xo, bp, k2, FIN_RNORM, dsc, slots + 6 * kMaxRhs, done, gate))) return q;
        if ((q = mp_update(dsc, c.m, 0, c.stream))) return q;
        return mp_load(S, rs, ps, r0s, r64, dsc, len, c.m, 0, c.ws, c.stream);
    };
    const int interval = c.opts.check_interval > 0 ? c.opts.check_interval : 8;
    cudaGraphExec_t exec = nullptr;
    if ((rc = capture(c, interval, iteration, &exec))) return rc;
    rc = run_graph(c, exec, dsc);
    cudaGraphExecDestroy(exec);
    if (rc) return rc;
    // x_e = b_e + kappa D_eo x_o (FP64)
    if ((rc = h64.launch(xe, xo, 0, EPI_XPAY, be, nullptr, c.kappa))) return rc;
    QCUB_CUDA_CHECK(cudaEventRecord(c.ev1, c.stream));
    if ((rc = finish_stats(c, D, g64, x, b, tmp64, slots))) return rc;
    for (int j = 0; j < c.m; ++j) {
        const double b2 = c.host_sc->bfull2[j];
        c.stats.recursive_residual[j] = b2 > 0 ? std::sqrt(c.host_sc->rtrue2[j] / b2) : 0.0;
    }
    float ms = 0.f;
    QCUB_CUDA_CHECK(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
    c.stats.solve_seconds = ms * 1e-3;
    if (c.stats.status != QCU_SUCCESS)
        return set_error(c.stats.status, "mixed BiCGStab stopped after %d iterations (%s)",
                         c.stats.iterations,
                         c.stats.status == QCU_ERR_BREAKDOWN ? "breakdown" : "max_iteration reached");
    return QCU_SUCCESS;
}

}  // namespace qcub
