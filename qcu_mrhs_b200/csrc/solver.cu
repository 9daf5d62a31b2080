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
//   stops only on the FP64 true residual.  A sloppy breakdown (non-finite or huge beta,
//   non-finite residual) restarts p and r0 from the FP64 residual at the next reliable
//   update; non-finite increments never reach x; and a FP64 residual that stops falling
//   ends the solve as not converged instead of running to max_iteration.
#include <cmath>
#include <cstring>
#include <functional>

#include "blas.h"
#include "context.h"
#include "dslash.h"
#include "precond.h"

namespace qcub {

namespace {

struct Hop {
    Context& c;
    int prec;
    const void* gauge;
    const void* links = nullptr;   // per-site tables of the tensor-core hop (or null)
    const uint32_t* nbr = nullptr;
    const int* active = nullptr;   // per-RHS activity flags (device), or null: all RHS
    // fetch (build on first use) the per-site tables when the hop kernel for this shape
    // reads them; call outside graph capture
    int tables() {
        if (!hop_reads_tables(c.nc, c.m, prec)) return QCU_SUCCESS;
        return c.hop_tables(prec, c.opts.t_boundary, &links, &nbr);
    }
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
        p.links = links;
        p.nbr = nbr;
        p.active = active;
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

// Capture `count` calls of body into *exec, reusing the executable graph *exec already
// holds when the new capture has its topology (cudaGraphExecUpdate copies every node's
// parameters from the new capture, so the result is the same as a fresh instantiation);
// otherwise, or when the update is refused, instantiate anew.  Saves the instantiation of
// the iteration block on every solve after the first of a context.
int capture_cached(Context& c, int count, const std::function<int()>& body, cudaGraphExec_t* exec) {
    if (!*exec) return capture(c, count, body, exec);
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
    cudaGraphExecUpdateResultInfo info{};
    if (cudaGraphExecUpdate(*exec, graph, &info) == cudaSuccess) {
        cudaGraphDestroy(graph);
        return QCU_SUCCESS;
    }
    cudaGetLastError();   // a refused update is not an error of this call
    cudaGraphExecDestroy(*exec);
    *exec = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
        *exec = nullptr;
        return set_error(QCU_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ei));
    }
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
    h.x_fresh = mixed;   // the sloppy increment starts from zero
    h.delta = c.opts.reliable_delta > 0 ? c.opts.reliable_delta : 0.1;
    h.quorum = c.opts.reliable_quorum > 0 ? (c.opts.reliable_quorum < 1 ? c.opts.reliable_quorum : 1.0) : 0.0;
    h.beta_max = mixed && c.opts.sloppy_precision == QCU_PRECISION_HALF ? kMaxHalfBeta : 1e300;
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

// alpha_j = rr_j / qq_j (0 for a finished or zero right-hand side)
__global__ void cg_alpha_kernel(double2* alpha, const double2* rr, const double2* qq, int m) {
    const int j = threadIdx.x;
    if (j >= m) return;
    alpha[j] = make_double2(qq[j].x > 0.0 ? rr[j].x / qq[j].x : 0.0, 0.0);
}

// beta_j = rr_new_j / rr_j ; rr_j <- rr_new_j
__global__ void cg_beta_kernel(double2* beta, double2* rr, const double2* rr_new, int m) {
    const int j = threadIdx.x;
    if (j >= m) return;
    beta[j] = make_double2(rr[j].x > 0.0 ? rr_new[j].x / rr[j].x : 0.0, 0.0);
    rr[j] = rr_new[j];
}

// recompute: the FP64 true residual from x (two hops); else (mixed solver) the FP64 residual
// of the last reliable update, which is the residual of the returned x up to the rounding
// of x_e = b_e + kappa D_eo x_o.
int finish_stats(Context& c, int prec, const void* gauge, const void* x, const void* b, void* tmp,
                 double2* slots, bool recompute = true) {
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
    if (!recompute) {
        for (int j = 0; j < c.m; ++j) {
            const double b2 = c.host_sc->bfull2[j];
            st.true_residual[j] = b2 > 0 ? std::sqrt(c.host_sc->rtrue2[j] / b2) : std::sqrt(c.host_sc->rtrue2[j]);
        }
        return QCU_SUCCESS;
    }
    return true_residual(c, prec, gauge, x, b, tmp, slots, st.true_residual);
}

}  // namespace

int SchurSolve::begin(void* x, const void* b, int max_iter, double tol) {
    x_ = static_cast<char*>(x);
    b_ = static_cast<const char*>(b);
    dsc_ = static_cast<BicgScalars*>(c_.scalars.ptr);
    return mixed_ ? begin_mixed(max_iter, tol) : begin_fused(max_iter, tol);
}

int SchurSolve::begin_fused(int max_iter, double tol) {
    Context& c = c_;
    P_ = c.in_prec;
    if (P_ != QCU_PRECISION_DOUBLE && P_ != QCU_PRECISION_SINGLE)
        return set_error(QCU_ERR_UNSUPPORTED, "the solve precision must be double or single");
    int rc = c.gauge_in(P_, &g_);
    if (rc) return rc;
    const size_t hb = c.half_bytes(P_);
    for (int i = 0; i < 8; ++i) {
        if ((rc = c.sv[i].ensure(hb))) return rc;
        v_[i] = c.sv[i].ptr;
    }
    if ((rc = c.sv[15].ensure(sizeof(double2) * 8 * kMaxRhs))) return rc;
    slots_ = static_cast<double2*>(c.sv[15].ptr);
    void* bp = v_[0];
    const void* be = b_;
    const void* bo = b_ + hb;
    const int64_t len = c.half_len();
    Hop hop{c, P_, g_};

    QCUB_CUDA_CHECK(cudaEventRecord(c.ev0, c.stream));
    if ((rc = prepare_scalars(c, dsc_, max_iter, tol, 0))) return rc;
    // b' = b_o + kappa D_oe b_e
    if ((rc = hop.launch(bp, be, 1, EPI_XPAY, bo, nullptr, c.kappa))) return rc;
    BicgStepArgs& a = a_;
    a.src = bp; a.r0 = v_[1]; a.r = v_[2]; a.p = v_[3]; a.v = v_[4]; a.s = v_[5]; a.t = v_[6];
    a.x = x_ + hb;
    a.sc = dsc_; a.ws = c.ws; a.len = len; a.m = c.m;
    if ((rc = bicg_step(STEP_INIT, P_, P_, a, c.stream))) return rc;
    // full-system norms of b (stopping reference with stop_true_residual)
    if ((rc = mrhs_dotc(slots_ + 4 * kMaxRhs, be, be, len, c.m, P_, c.ws, c.stream))) return rc;
    if ((rc = mrhs_dotc(slots_ + 5 * kMaxRhs, bo, bo, len, c.m, P_, c.ws, c.stream))) return rc;
    set_bfull_kernel<<<1, 64, 0, c.stream>>>(dsc_, slots_ + 4 * kMaxRhs, slots_ + 5 * kMaxRhs, c.m,
                                             c.opts.stop_true_residual ? 1 : 0);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

int SchurSolve::begin_mixed(int max_iter, double tol) {
    Context& c = c_;
    if (c.in_prec != QCU_PRECISION_DOUBLE)
        return set_error(QCU_ERR_UNSUPPORTED, "mixed precision needs double-precision fields");
    S_ = c.opts.sloppy_precision;
    if (S_ != QCU_PRECISION_SINGLE && S_ != QCU_PRECISION_HALF && S_ != QCU_PRECISION_BF16)
        return set_error(QCU_ERR_INVALID, "sloppy precision %d (single, half or bf16)", S_);
    P_ = QCU_PRECISION_DOUBLE;
    int rc;
    if ((rc = c.gauge_in(P_, &g_))) return rc;
    if ((rc = c.gauge_in(S_, &gs_))) return rc;
    {   // the sloppy hop's per-site tables, built here, before the iterations are captured
        Hop t{c, S_, gs_};
        if ((rc = t.tables())) return rc;
        links_s_ = t.links;
        nbr_s_ = t.nbr;
    }
    const size_t hb = c.half_bytes(P_);
    const size_t hs = c.half_bytes(S_);
    const size_t he = c.half_bytes(QCU_PRECISION_SINGLE);
    for (int i = 0; i < 11; ++i) {
        if ((rc = c.sv[i].ensure(i < 3 ? hb : (i < 10 ? hs : he)))) return rc;
        v_[i] = c.sv[i].ptr;
    }
    if ((rc = c.sv[15].ensure(sizeof(double2) * 8 * kMaxRhs))) return rc;
    slots_ = static_cast<double2*>(c.sv[15].ptr);
    // v_: 0 b', 1 r64, 2 tmp64, 3 r0s, 4 rs, 5 ps, 6 vs, 7 ss, 8 ts, 9 tmps, 10 e (FP32)
    void* bp = v_[0];
    void* r64 = v_[1];
    const void* be = b_;
    const void* bo = b_ + hb;
    void* xo = x_ + hb;
    const int64_t len = c.half_len();
    Hop h64{c, P_, g_};

    QCUB_CUDA_CHECK(cudaEventRecord(c.ev0, c.stream));
    if ((rc = prepare_scalars(c, dsc_, max_iter, tol, 1))) return rc;
    // b' = b_o + kappa D_oe b_e (FP64); ||b||^2 of the full system
    if ((rc = h64.launch(bp, be, 1, EPI_XPAY, bo, nullptr, c.kappa))) return rc;
    if ((rc = mrhs_dotc(slots_ + 4 * kMaxRhs, be, be, len, c.m, P_, c.ws, c.stream))) return rc;
    if ((rc = mrhs_dotc(slots_ + 5 * kMaxRhs, bo, bo, len, c.m, P_, c.ws, c.stream))) return rc;
    set_bfull_kernel<<<1, 64, 0, c.stream>>>(dsc_, slots_ + 4 * kMaxRhs, slots_ + 5 * kMaxRhs, c.m, 1);
    QCUB_CHECK_LAUNCH();
    // x_o = 0, r64 = b', rtrue2 = ||b'||^2 (the increment e starts from zero through x_fresh)
    QCUB_CUDA_CHECK(cudaMemsetAsync(xo, 0, hb, c.stream));
    QCUB_CUDA_CHECK(cudaMemcpyAsync(r64, bp, hb, cudaMemcpyDeviceToDevice, c.stream));
    if ((rc = mrhs_norm(nullptr, r64, len, c.m, P_, c.ws, c.stream, FIN_RNORM, dsc_))) return rc;
    if ((rc = mp_update(dsc_, c.m, 1, c.stream))) return rc;
    if ((rc = mp_load(S_, v_[4], v_[5], v_[3], r64, dsc_, len, c.m, 1, c.ws, c.stream))) return rc;
    BicgStepArgs& a = a_;
    a.r0 = v_[3]; a.r = v_[4]; a.p = v_[5]; a.v = v_[6]; a.s = v_[7]; a.t = v_[8]; a.x = v_[10];
    a.sc = dsc_; a.ws = c.ws; a.len = len; a.m = c.m;
    return QCU_SUCCESS;
}

int SchurSolve::enqueue_iteration() {
    Context& c = c_;
    const double k2 = c.kappa * c.kappa;
    const int* done = &dsc_->done;
    int e;
    if (!mixed_) {
        void* r0 = v_[1]; void* p = v_[3]; void* v = v_[4]; void* s = v_[5]; void* t = v_[6];
        void* tmp = v_[7];
        Hop hop{c, P_, g_};
        if ((e = hop.launch(tmp, p, 0, EPI_PLAIN, nullptr, nullptr, 0.0, FIN_NONE, nullptr, nullptr, done))) return e;
        if ((e = hop.launch(v, tmp, 1, EPI_SCHUR_R0, p, r0, k2, FIN_ALPHA, dsc_, dsc_->red[0], done))) return e;
        if ((e = bicg_step(STEP_S, P_, P_, a_, c.stream))) return e;
        if ((e = hop.launch(tmp, s, 0, EPI_PLAIN, nullptr, nullptr, 0.0, FIN_NONE, nullptr, nullptr, done))) return e;
        if ((e = hop.launch(t, tmp, 1, EPI_SCHUR_TS, s, nullptr, k2, FIN_OMEGA, dsc_, dsc_->red[0], done))) return e;
        if ((e = bicg_step(STEP_XR, P_, P_, a_, c.stream))) return e;
        return bicg_step(STEP_P, P_, P_, a_, c.stream);
    }
    void* bp = v_[0]; void* r64 = v_[1]; void* tmp64 = v_[2];
    void* r0s = v_[3]; void* rs = v_[4]; void* ps = v_[5]; void* vs = v_[6]; void* ss = v_[7];
    void* ts = v_[8]; void* tmps = v_[9]; void* ev = v_[10];
    void* xo = x_ + c.half_bytes(P_);
    const int64_t len = c.half_len();
    const int* gate = &dsc_->gate;
    const int XP = QCU_PRECISION_SINGLE;
    Hop h64{c, P_, g_};
    // sloppy hops skip the groups of 4 RHS whose FP64 residual has converged: the reliable
    // update clears their flags, their scalars are 0 from then on, so their sloppy vectors
    // keep finite values that no update uses
    Hop hs{c, S_, gs_, links_s_, nbr_s_, dsc_->active};
    // sloppy BiCGStab iteration
    if ((e = hs.launch(tmps, ps, 0, EPI_PLAIN, nullptr, nullptr, 0.0, FIN_NONE, nullptr, nullptr, done))) return e;
    if ((e = hs.launch(vs, tmps, 1, EPI_SCHUR_R0, ps, r0s, k2, FIN_ALPHA, dsc_, dsc_->red[0], done))) return e;
    if ((e = bicg_step(STEP_S, S_, XP, a_, c.stream))) return e;
    if ((e = hs.launch(tmps, ss, 0, EPI_PLAIN, nullptr, nullptr, 0.0, FIN_NONE, nullptr, nullptr, done))) return e;
    if ((e = hs.launch(ts, tmps, 1, EPI_SCHUR_TS, ss, nullptr, k2, FIN_OMEGA, dsc_, dsc_->red[0], done))) return e;
    if ((e = bicg_step(STEP_XR, S_, XP, a_, c.stream))) return e;
    if ((e = bicg_step(STEP_P, S_, XP, a_, c.stream))) return e;
    // reliable update (every kernel returns at once unless one is pending)
    if ((e = mp_accum(xo, ev, dsc_, len, c.m, c.stream))) return e;
    if ((e = h64.launch(tmp64, xo, 0, EPI_PLAIN, nullptr, nullptr, 0.0, FIN_NONE, nullptr, nullptr, done, gate))) return e;
    if ((e = h64.launch(r64, tmp64, 1, EPI_RESID, xo, bp, k2, FIN_RNORM, dsc_, slots_ + 6 * kMaxRhs, done, gate))) return e;
    if ((e = mp_update(dsc_, c.m, 0, c.stream))) return e;
    return mp_load(S_, rs, ps, r0s, r64, dsc_, len, c.m, 0, c.ws, c.stream);
}

int SchurSolve::end() {
    Context& c = c_;
    int rc;
    const size_t hb = c.half_bytes(P_);
    void* tmp = mixed_ ? v_[2] : v_[7];
    // final device scalars (iterations, status, norms) for the statistics
    QCUB_CUDA_CHECK(cudaMemcpyAsync(c.host_sc, dsc_, sizeof(BicgScalars), cudaMemcpyDeviceToHost, c.stream));
    QCUB_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    Hop hop{c, P_, g_};
    // x_e = b_e + kappa D_eo x_o
    if ((rc = hop.launch(x_, x_ + hb, 0, EPI_XPAY, b_, nullptr, c.kappa))) return rc;
    QCUB_CUDA_CHECK(cudaEventRecord(c.ev1, c.stream));
    if ((rc = finish_stats(c, P_, g_, x_, b_, tmp, slots_, !mixed_))) return rc;
    if (mixed_)
        for (int j = 0; j < c.m; ++j) {
            const double b2 = c.host_sc->bfull2[j];
            c.stats.recursive_residual[j] = b2 > 0 ? std::sqrt(c.host_sc->rtrue2[j] / b2) : 0.0;
        }
    float ms = 0.f;
    QCUB_CUDA_CHECK(cudaEventSynchronize(c.ev1));
    QCUB_CUDA_CHECK(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
    c.stats.solve_seconds = ms * 1e-3;
    if (c.stats.status != QCU_SUCCESS)
        return set_error(c.stats.status, "%sBiCGStab stopped after %d iterations (%s)", mixed_ ? "mixed " : "",
                         c.stats.iterations,
                         c.stats.status == QCU_ERR_BREAKDOWN ? "breakdown"
                         : c.host_sc->status == 4           ? "the FP64 residual stagnated"
                                                            : "max_iteration reached");
    return QCU_SUCCESS;
}

namespace {

int solve_one(Context& c, void* x, const void* b, int max_iter, double tol, bool mixed) {
    SchurSolve solve(c, mixed);
    int rc = solve.begin(x, b, max_iter, tol);
    if (rc) return rc;
    const int interval = c.opts.check_interval > 0 ? c.opts.check_interval : 8;
    if ((rc = capture_cached(c, interval, [&]() { return solve.enqueue_iteration(); }, &c.iter_exec))) return rc;
    if ((rc = run_graph(c, c.iter_exec, solve.device_scalars()))) return rc;
    return solve.end();
}

}  // namespace

int solve_fused(Context& c, void* x, const void* b, int max_iter, double tol) {
    return solve_one(c, x, b, max_iter, tol, false);
}

int solve_mixed(Context& c, void* x, const void* b, int max_iter, double tol) {
    return solve_one(c, x, b, max_iter, tol, true);
}

// CGNR on the even/odd Schur system: conjugate gradients on A^dag A x_o = A^dag b'_o with
// A = 1 - kappa^2 D_oe D_eo and A^dag = 1 - kappa^2 (D^dag)_oe (D^dag)_eo (the dagger hops).
// The Schur residual s = b' - A x_o is carried along (s -= alpha A p), so the stopping rules
// are those of the BiCGStab solvers: ||s_j|| <= tol ||b'_j|| for every RHS, or the
// full-system ||b_j|| with stop_true_residual.  The host reads the residual norms every
// iteration.
int solve_cgnr(Context& c, void* x, const void* b, int max_iter, double tol) {
    const int P = c.in_prec;
    if (P != QCU_PRECISION_DOUBLE && P != QCU_PRECISION_SINGLE)
        return set_error(QCU_ERR_UNSUPPORTED, "the CGNR solve needs double or single precision fields");
    const void* g = nullptr;
    int rc;
    if ((rc = c.gauge_in(P, &g))) return rc;
    const size_t hb = c.half_bytes(P);
    void* v_[7];
    for (int i = 0; i < 7; ++i) {
        if ((rc = c.sv[i].ensure(hb))) return rc;
        v_[i] = c.sv[i].ptr;
    }
    if ((rc = c.sv[15].ensure(sizeof(double2) * 8 * kMaxRhs))) return rc;
    double2* sl = static_cast<double2*>(c.sv[15].ptr);
    double2 *rr = sl, *qq = sl + kMaxRhs, *alpha = sl + 2 * kMaxRhs, *beta = sl + 3 * kMaxRhs;
    double2 *rrn = sl + 4 * kMaxRhs, *ss = sl + 5 * kMaxRhs, *bb = sl + 6 * kMaxRhs, *be2 = sl + 7 * kMaxRhs;
    void* bp = v_[0]; void* sres = v_[1]; void* r = v_[2]; void* p = v_[3]; void* qv = v_[4]; void* z = v_[5];
    void* tmp = v_[6];
    const char* be = static_cast<const char*>(b);
    const void* bo = be + hb;
    char* xe = static_cast<char*>(x);
    void* xo = xe + hb;
    const int64_t len = c.half_len();
    const int m = c.m;
    const double k2 = c.kappa * c.kappa;
    const cudaStream_t st = c.stream;
    auto hop = [&](void* out, const void* in, int parity, bool dag, int epi, const void* xv, double a) -> int {
        HopParams hp{};
        hp.out = out; hp.in = in; hp.gauge = g; hp.x = xv; hp.a = a;
        hp.g = c.g; hp.m = m; hp.parity = parity; hp.t_sign = c.opts.t_boundary;
        hp.red = RedArgs{c.ws.partials, c.ws.counter, c.ws.result, nullptr, nullptr, FIN_NONE};
        return hop_launch(hp, c.nc, P, dag, epi, st);
    };
    // A v (dag = false) or A^dag v (dag = true) into out, through tmp
    auto schur = [&](void* out, const void* in, bool dag) -> int {
        int e;
        if ((e = hop(tmp, in, 0, dag, EPI_PLAIN, nullptr, 0.0))) return e;
        return hop(out, tmp, 1, dag, EPI_XPAY, in, -k2);
    };
    QCUB_CUDA_CHECK(cudaEventRecord(c.ev0, st));
    // b' = b_o + kappa D_oe b_e ; s = b' ; r = p = A^dag b' ; x_o = 0
    if ((rc = hop(bp, be, 1, false, EPI_XPAY, bo, c.kappa))) return rc;
    QCUB_CUDA_CHECK(cudaMemcpyAsync(sres, bp, hb, cudaMemcpyDeviceToDevice, st));
    if ((rc = schur(r, bp, true))) return rc;
    QCUB_CUDA_CHECK(cudaMemcpyAsync(p, r, hb, cudaMemcpyDeviceToDevice, st));
    QCUB_CUDA_CHECK(cudaMemsetAsync(xo, 0, hb, st));
    if ((rc = mrhs_dotc(rr, r, r, len, m, P, c.ws, st))) return rc;
    if ((rc = mrhs_dotc(bb, bp, bp, len, m, P, c.ws, st))) return rc;
    if ((rc = mrhs_dotc(be2, be, be, len, m, P, c.ws, st))) return rc;
    if ((rc = mrhs_dotc(qq, bo, bo, len, m, P, c.ws, st))) return rc;   // ||b_o||^2, reused below
    double2 h[3 * kMaxRhs];
    QCUB_CUDA_CHECK(cudaMemcpyAsync(h, bb, sizeof(double2) * kMaxRhs, cudaMemcpyDeviceToHost, st));
    QCUB_CUDA_CHECK(cudaMemcpyAsync(h + kMaxRhs, be2, sizeof(double2) * kMaxRhs, cudaMemcpyDeviceToHost, st));
    QCUB_CUDA_CHECK(cudaMemcpyAsync(h + 2 * kMaxRhs, qq, sizeof(double2) * kMaxRhs, cudaMemcpyDeviceToHost, st));
    QCUB_CUDA_CHECK(cudaStreamSynchronize(st));
    double ref2[kMaxRhs];   // stopping reference ||b'||^2 or ||b||^2 per RHS
    for (int j = 0; j < m; ++j)
        ref2[j] = c.opts.stop_true_residual ? h[kMaxRhs + j].x + h[2 * kMaxRhs + j].x : h[j].x;
    int it = 0, status = 3;
    double sn2[kMaxRhs];
    for (int j = 0; j < m; ++j) sn2[j] = h[j].x;
    auto converged = [&]() {
        for (int j = 0; j < m; ++j)
            if (sn2[j] > tol * tol * ref2[j]) return false;
        return true;
    };
    if (converged()) status = 1;
    while (status == 3 && it < max_iter) {
        if ((rc = schur(qv, p, false))) return rc;       // q = A p
        if ((rc = schur(z, qv, true))) return rc;        // z = A^dag q
        if ((rc = mrhs_dotc(qq, qv, qv, len, m, P, c.ws, st))) return rc;
        cg_alpha_kernel<<<1, kMaxRhs, 0, st>>>(alpha, rr, qq, m);
        QCUB_CHECK_LAUNCH();
        if ((rc = mrhs_axpy(OP_XPAY, xo, alpha, xo, nullptr, p, nullptr, nullptr, len, m, P, st))) return rc;
        if ((rc = mrhs_axpy(OP_XSAY, sres, alpha, sres, nullptr, qv, nullptr, nullptr, len, m, P, st))) return rc;
        if ((rc = mrhs_axpy(OP_XSAY, r, alpha, r, nullptr, z, nullptr, nullptr, len, m, P, st))) return rc;
        if ((rc = mrhs_dotc(rrn, r, r, len, m, P, c.ws, st))) return rc;
        cg_beta_kernel<<<1, kMaxRhs, 0, st>>>(beta, rr, rrn, m);
        QCUB_CHECK_LAUNCH();
        if ((rc = mrhs_axpy(OP_XPAY, p, beta, r, nullptr, p, nullptr, nullptr, len, m, P, st))) return rc;
        if ((rc = mrhs_dotc(ss, sres, sres, len, m, P, c.ws, st))) return rc;
        QCUB_CUDA_CHECK(cudaMemcpyAsync(h, ss, sizeof(double2) * kMaxRhs, cudaMemcpyDeviceToHost, st));
        QCUB_CUDA_CHECK(cudaStreamSynchronize(st));
        ++it;
        for (int j = 0; j < m; ++j) sn2[j] = h[j].x;
        bool finite = true;
        for (int j = 0; j < m; ++j) finite = finite && std::isfinite(sn2[j]);
        if (!finite) status = 2;
        else if (converged()) status = 1;
    }
    // x_e = b_e + kappa D_eo x_o
    if ((rc = hop(xe, xo, 0, false, EPI_XPAY, be, c.kappa))) return rc;
    QCUB_CUDA_CHECK(cudaEventRecord(c.ev1, st));
    c.host_sc->iter = it;
    c.host_sc->reliable = 0;
    c.host_sc->status = status;
    for (int j = 0; j < m; ++j) {
        c.host_sc->bnorm2[j] = ref2[j];
        c.host_sc->rnorm2[j] = sn2[j];
    }
    if ((rc = finish_stats(c, P, g, x, b, tmp, sl))) return rc;
    float ms = 0.f;
    QCUB_CUDA_CHECK(cudaEventSynchronize(c.ev1));
    QCUB_CUDA_CHECK(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
    c.stats.solve_seconds = ms * 1e-3;
    if (c.stats.status != QCU_SUCCESS)
        return set_error(c.stats.status, "CGNR stopped after %d iterations (%s)", it,
                         c.stats.status == QCU_ERR_BREAKDOWN ? "breakdown" : "max_iteration reached");
    return QCU_SUCCESS;
}

// Right-preconditioned BiCGStab on the full system M (P y) = b, x = P y, in FP64 with P
// applied in FP32 (x and r are updated with the P outputs actually computed, so the
// recursive residual stays the FP64 residual of x whatever P's rounding).  Stops when
// every RHS has ||r_j|| <= tol ||b_j|| on the full system.  When it breaks down or hits
// max_iter, the plain FP64 Schur BiCGStab solves the system instead.
int solve_precond(Context& c, Precond* P, void* x, const void* b, int max_iter, double tol) {
    if (!P) return set_error(QCU_ERR_STATE, "no preconditioner attached (qcuSetPreconditioner)");
    if (c.in_prec != QCU_PRECISION_DOUBLE)
        return set_error(QCU_ERR_UNSUPPORTED, "the preconditioned solve needs double-precision fields");
    for (int i = 0; i < 4; ++i)
        if (P->g.L[i] != c.g.L[i]) return set_error(QCU_ERR_INVALID, "preconditioner lattice differs");
    if (P->nc != c.nc || P->m != c.m) return set_error(QCU_ERR_INVALID, "preconditioner n_color / m_rhs differ");
    if (P->t_sign != c.opts.t_boundary) return set_error(QCU_ERR_INVALID, "preconditioner t boundary differs");
    const int D = QCU_PRECISION_DOUBLE, F = QCU_PRECISION_SINGLE;
    const void* g64 = nullptr;
    const void* g32 = nullptr;
    int rc;
    if ((rc = c.gauge_in(D, &g64)) || (rc = c.gauge_in(F, &g32))) return rc;
    const size_t fb = 2 * c.half_bytes(D), ff = 2 * c.half_bytes(F);
    void* v_[10];
    for (int i = 0; i < 10; ++i) {
        if ((rc = c.sv[i].ensure(i < 8 ? fb : ff))) return rc;
        v_[i] = c.sv[i].ptr;
    }
    if ((rc = c.sv[15].ensure(sizeof(double2) * 8 * kMaxRhs))) return rc;
    double2* slots = static_cast<double2*>(c.sv[15].ptr);
    void* r0 = v_[0]; void* r = v_[1]; void* p = v_[2]; void* v = v_[3]; void* s = v_[4]; void* t = v_[5];
    void* ph = v_[6]; void* sh = v_[7];
    float2* fin = static_cast<float2*>(v_[8]);
    float2* fout = static_cast<float2*>(v_[9]);
    BicgScalars* dsc = static_cast<BicgScalars*>(c.scalars.ptr);
    const int64_t len = 2 * c.half_len();
    const int64_t n = len * c.m;
    const int* done = &dsc->done;

    QCUB_CUDA_CHECK(cudaEventRecord(c.ev0, c.stream));
    if ((rc = prepare_scalars(c, dsc, max_iter, tol, 0))) return rc;
    BicgStepArgs a;
    a.src = const_cast<void*>(b); a.r0 = r0; a.r = r; a.p = p; a.v = v; a.s = s; a.t = t; a.x = x;
    a.sc = dsc; a.ws = c.ws; a.len = len; a.m = c.m;
    if ((rc = bicg_step(STEP_INIT, D, D, a, c.stream))) return rc;
    auto precondition = [&](void* out64, const void* in64) -> int {
        int e;
        if ((e = pc_cast(fin, F, in64, D, n, done, c.stream))) return e;
        if ((e = P->apply(fout, fin, g32, c.stream, done))) return e;
        return pc_cast(out64, D, fout, F, n, done, c.stream);
    };
    auto iteration = [&]() -> int {
        int e;
        if ((e = precondition(ph, p))) return e;
        if ((e = full_mat(v, ph, g64, c.g, c.nc, c.m, c.kappa, c.opts.t_boundary, false, D, c.stream, done))) return e;
        if ((e = pc_alpha(r0, v, dsc, len, c.m, c.ws, c.stream))) return e;
        if ((e = bicg_step(STEP_S, D, D, a, c.stream))) return e;
        if ((e = precondition(sh, s))) return e;
        if ((e = full_mat(t, sh, g64, c.g, c.nc, c.m, c.kappa, c.opts.t_boundary, false, D, c.stream, done))) return e;
        if ((e = pc_omega(t, s, dsc, len, c.m, c.ws, c.stream))) return e;
        if ((e = pc_xr(x, r, ph, sh, s, t, r0, dsc, len, c.m, c.ws, c.stream))) return e;
        return bicg_step(STEP_P, D, D, a, c.stream);
    };
    const int interval = c.opts.check_interval > 0 ? c.opts.check_interval : 8;
    cudaGraphExec_t exec = nullptr;
    if ((rc = capture(c, interval, iteration, &exec))) return rc;
    rc = run_graph(c, exec, dsc);
    cudaGraphExecDestroy(exec);
    if (rc) return rc;
    QCUB_CUDA_CHECK(cudaEventRecord(c.ev1, c.stream));
    if ((rc = finish_stats(c, D, g64, x, b, v, slots))) return rc;
    float ms = 0.f;
    QCUB_CUDA_CHECK(cudaEventSynchronize(c.ev1));
    QCUB_CUDA_CHECK(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
    c.stats.solve_seconds = ms * 1e-3;
    c.stats.precond_iterations = c.stats.iterations;
    if (c.stats.status == QCU_SUCCESS) return QCU_SUCCESS;
    // fallback: the plain FP64 Schur BiCGStab from scratch
    const int pit = c.stats.iterations;
    const double pre_seconds = c.stats.solve_seconds;
    c.stats = QcuSolveStats{};
    rc = solve_fused(c, x, b, max_iter, tol);
    c.stats.fallback = 1;
    c.stats.precond_iterations = pit;
    c.stats.solve_seconds += pre_seconds;
    return rc;
}

}  // namespace qcub
