// batch.cu -- many independent Schur BiCGStab solves (each with its own lattice, colour
// count, RHS count, kappa, tolerance and gauge field) advanced together on one GPU.
//
// Every system gets its own context (stream, reduction scratch, device scalars, solver
// vectors).  The iterations of all systems are captured into ONE CUDA graph in which each
// system is an independent branch, so the small kernels of small lattices run side by
// side and fill the SMs that one small system leaves idle.
//
// Two drivers of that graph:
//   device loop (default): each branch is a conditional WHILE node whose body holds
//     `check_interval` iterations plus a control kernel; the control kernel ends the loop
//     once the system's device scalars say `done` (converged, breakdown or max_iteration)
//     and stamps the device clock at that moment.  The whole batch runs as one graph launch
//     with no host round trip; a converged system's branch stops, the others go on.
//     The loop is bounded twice: the finisher sets `done` at max_iteration, and the control
//     kernel also ends it after ceil(max_iteration / check_interval) + 2 passes.
//   host loop (QCU_BATCH_HOST_LOOP): each branch holds `check_interval` iterations; the host
//     relaunches the graph and reads every system's `done` flag between launches
//     (converged systems' kernels return at once).
// Converged right-hand sides inside a running system are frozen with freeze_converged (on
// when no options are given); the mixed solver's sloppy hops skip their groups of 4 RHS.
// Before capture, the hop kernel of every distinct (n_color, m_rhs, precision) is picked
// by the autotuner (tune.cu) unless one is already recorded.
#include <chrono>
#include <cmath>
#include <memory>
#include <mutex>
#include <vector>

#include "blas.h"
#include "context.h"
#include "dslash.h"
#include "layout.h"

namespace qcub {

int tune_hop(const int L[4], int nc, int m, int prec, cudaStream_t st, double* best_us);
int tuned_hop(int nc, int m, int prec);
int hop_kind();
const char* last_message();

namespace {

constexpr int kMaxBatch = 1024;

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__global__ void batch_stamp_kernel(unsigned long long* t) { *t = global_ns(); }

// End of one WHILE-loop pass of system `i`: stop the loop when the solve is done or the
// pass limit is reached, and stamp the device clock the first time.
__global__ void batch_loop_kernel(cudaGraphConditionalHandle h, const BicgScalars* sc, unsigned* passes,
                                  unsigned limit, unsigned long long* stamp) {
    const unsigned k = ++*passes;
    if (sc->done || k >= limit) {
        if (*stamp == 0ull) *stamp = global_ns();
        cudaGraphSetConditional(h, 0);
    }
}

// Contexts kept by QCU_BATCH_KEEP_CONTEXTS for later batches (their device buffers stay
// allocated, which saves the first-touch cost of fresh device memory on every call).
std::mutex g_cache_mu;
std::vector<Context*> g_cache;

Context* cache_take(const int L[4], int nc, int m) {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    for (size_t i = 0; i < g_cache.size(); ++i) {
        Context* c = g_cache[i];
        if (c->g.L[0] == L[0] && c->g.L[1] == L[1] && c->g.L[2] == L[2] && c->g.L[3] == L[3] && c->nc == nc &&
            c->m == m) {
            g_cache.erase(g_cache.begin() + (long)i);
            return c;
        }
    }
    return nullptr;
}

void cache_put(Context* c) {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    g_cache.push_back(c);
}

struct System {
    Context* c = nullptr;
    bool keep = false;   // return the context to the cache instead of destroying it
    std::unique_ptr<SchurSolve> solve;
    ~System() {
        solve.reset();
        if (keep && c) cache_put(c);
        else context_destroy(c);
    }
};

struct BatchState {
    std::vector<std::unique_ptr<System>> sys;
    cudaStream_t master = nullptr;
    cudaEvent_t fork = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned* d_passes = nullptr;               // [n]
    unsigned long long* d_stamp = nullptr;      // [n + 1]: done stamps, start stamp at [n]
    int* h_done = nullptr;                      // pinned [n]
    ~BatchState() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (master) cudaStreamSynchronize(master);
        if (d_passes) cudaFree(d_passes);
        if (d_stamp) cudaFree(d_stamp);
        if (h_done) cudaFreeHost(h_done);
        if (fork) cudaEventDestroy(fork);
        if (master) cudaStreamDestroy(master);
        sys.clear();
    }
};

int validate(const QcuBatchSystem& s, int i) {
    if (!s.gauge || !s.b || !s.x) return set_error(QCU_ERR_INVALID, "system %d: null pointer", i);
    if (!(s.kappa > 0.0) || !(s.tol > 0.0))
        return set_error(QCU_ERR_INVALID, "system %d: kappa %g, tol %g", i, s.kappa, s.tol);
    for (int j = 0; j < s.m_rhs && j < kMaxRhs; ++j)
        if (!s.b[j] || !s.x[j]) return set_error(QCU_ERR_INVALID, "system %d: null fermion %d", i, j);
    return QCU_SUCCESS;
}

// gather (scatter) the m full-lattice caller fields of a system into (out of) its
// gathered buffer, even half first
int move_fields(Context& c, void* const* ptrs, void* gathered, bool gather) {
    const int P = c.in_prec;
    const size_t hb = c.half_bytes(P);
    const size_t half_ext = (size_t)c.g.vh * 4 * c.nc * 2 * prec_bytes(P);
    void* per[kMaxRhs];
    for (int par = 0; par < 2; ++par) {
        for (int j = 0; j < c.m; ++j) per[j] = static_cast<char*>(ptrs[j]) + par * half_ext;
        char* g = static_cast<char*>(gathered) + par * hb;
        const int rc = gather ? gather_mrhs(g, P, per, P, c.g.vh, c.nc, c.m, c.stream)
                              : scatter_mrhs(per, P, g, P, c.g.vh, c.nc, c.m, c.stream);
        if (rc) return rc;
    }
    return QCU_SUCCESS;
}

int autotune(const std::vector<std::unique_ptr<System>>& sys, const QcuSolverOptions& o, cudaStream_t st) {
    if (hop_kind() != QCU_HOP_AUTO) return QCU_SUCCESS;   // a fixed kernel was requested
    for (const auto& s : sys) {
        const Context& c = *s->c;
        int precs[2] = {c.in_prec, o.solver == QCU_SOLVER_MIXED ? o.sloppy_precision : -1};
        for (int prec : precs) {
            if (prec < 0 || tuned_hop(c.nc, c.m, prec) > 0) continue;
            const int r = tune_hop(c.g.L, c.nc, c.m, prec, st, nullptr);
            if (r < 0) return -r;
        }
    }
    return QCU_SUCCESS;
}

int capture_device_loop(BatchState& bs, int interval) {
    const int n = (int)bs.sys.size();
    QCUB_CUDA_CHECK(cudaGraphCreate(&bs.graph, 0));
    for (int i = 0; i < n; ++i) {
        Context& c = *bs.sys[i]->c;
        cudaGraphConditionalHandle h;
        QCUB_CUDA_CHECK(cudaGraphConditionalHandleCreate(&h, bs.graph, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        QCUB_CUDA_CHECK(cudaGraphAddNode(&node, bs.graph, nullptr, 0, &np));
        cudaGraph_t body = np.conditional.phGraph_out[0];
        QCUB_CUDA_CHECK(
            cudaStreamBeginCaptureToGraph(c.stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        int rc = QCU_SUCCESS;
        for (int k = 0; k < interval && rc == QCU_SUCCESS; ++k) rc = bs.sys[i]->solve->enqueue_iteration();
        const BicgScalars* dsc = bs.sys[i]->solve->device_scalars();
        const unsigned limit = (unsigned)((c.host_sc->max_iter + interval - 1) / interval + 2);
        if (rc == QCU_SUCCESS) {
            batch_loop_kernel<<<1, 1, 0, c.stream>>>(h, dsc, bs.d_passes + i, limit, bs.d_stamp + i);
            const cudaError_t le = cudaGetLastError();
            if (le != cudaSuccess) rc = set_error(QCU_ERR_CUDA, "loop kernel: %s", cudaGetErrorString(le));
        }
        cudaGraph_t out = nullptr;
        const cudaError_t e = cudaStreamEndCapture(c.stream, &out);
        if (rc) return rc;
        if (e != cudaSuccess) return set_error(QCU_ERR_CUDA, "body capture: %s", cudaGetErrorString(e));
    }
    const cudaError_t ei = cudaGraphInstantiate(&bs.exec, bs.graph, 0);
    if (ei != cudaSuccess) return set_error(QCU_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ei));
    return QCU_SUCCESS;
}

int capture_host_loop(BatchState& bs, int interval) {
    const int n = (int)bs.sys.size();
    QCUB_CUDA_CHECK(cudaStreamBeginCapture(bs.master, cudaStreamCaptureModeThreadLocal));
    int rc = QCU_SUCCESS;
    cudaError_t e = cudaEventRecord(bs.fork, bs.master);
    for (int i = 0; i < n && rc == QCU_SUCCESS && e == cudaSuccess; ++i) {
        Context& c = *bs.sys[i]->c;
        e = cudaStreamWaitEvent(c.stream, bs.fork, 0);
        for (int k = 0; k < interval && rc == QCU_SUCCESS && e == cudaSuccess; ++k)
            rc = bs.sys[i]->solve->enqueue_iteration();
        if (e == cudaSuccess) e = cudaEventRecord(c.ev_in, c.stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(bs.master, c.ev_in, 0);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(bs.master, &g);
    if (g) bs.graph = g;
    if (rc) return rc;
    if (e != cudaSuccess || ee != cudaSuccess)
        return set_error(QCU_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e != cudaSuccess ? e : ee));
    const cudaError_t ei = cudaGraphInstantiate(&bs.exec, bs.graph, 0);
    if (ei != cudaSuccess) return set_error(QCU_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ei));
    return QCU_SUCCESS;
}

int invert_batch(QcuBatchSystem* sys, int n, const QcuSolverOptions* opts_in, int flags) {
    if (!sys || n < 1 || n > kMaxBatch) return set_error(QCU_ERR_INVALID, "batch of %d systems (1..%d)", n, kMaxBatch);
    QcuSolverOptions o{};
    if (opts_in) {
        o = *opts_in;
    } else {
        qcuGetDefaultSolverOptions(&o);
        o.freeze_converged = 1;   // batch default: converged RHS stop (and drop out of the hops)
    }
    if (o.solver < QCU_SOLVER_REFERENCE || o.solver > QCU_SOLVER_MIXED)
        return set_error(QCU_ERR_INVALID, "solver %d", o.solver);
    if (o.t_boundary != 1.0 && o.t_boundary != -1.0) return set_error(QCU_ERR_INVALID, "t_boundary must be +1 or -1");
    const bool mixed = o.solver == QCU_SOLVER_MIXED;
    const int interval = o.check_interval > 0 ? o.check_interval : 8;
    int rc;
    for (int i = 0; i < n; ++i) {
        if ((rc = validate(sys[i], i))) return rc;
        sys[i].iterations = 0;
        sys[i].reliable_updates = 0;
        sys[i].status = QCU_ERR_STATE;
        sys[i].true_residual_max = 0.0;
        sys[i].latency_seconds = 0.0;
    }

    BatchState bs;
    for (int i = 0; i < n; ++i) {
        auto s = std::make_unique<System>();
        s->keep = (flags & QCU_BATCH_KEEP_CONTEXTS) != 0;
        s->c = s->keep ? cache_take(sys[i].lattice_size, sys[i].n_color, sys[i].m_rhs) : nullptr;
        if (!s->c) {
            s->c = new Context();
            if ((rc = context_init(s->c, sys[i].lattice_size, sys[i].n_color, sys[i].m_rhs, QCU_PRECISION_DOUBLE,
                                   QCU_PRECISION_DOUBLE))) {
                s->keep = false;
                return set_error(rc, "system %d: %s", i, last_message());
            }
        }
        Context& c = *s->c;
        c.opts = o;
        c.precond = nullptr;
        c.kappa = sys[i].kappa;
        c.mass = 1.0 / (2.0 * sys[i].kappa) - 4.0;
        c.dslash_ready = true;
        if ((rc = context_load_gauge(&c, sys[i].gauge, QCU_PRECISION_DOUBLE))) return rc;
        const size_t hb = c.half_bytes(c.in_prec);
        if ((rc = c.mrhs_in.ensure(2 * hb)) || (rc = c.mrhs_out.ensure(2 * hb))) return rc;
        if ((rc = move_fields(c, sys[i].b, c.mrhs_in.ptr, true))) return rc;
        bs.sys.push_back(std::move(s));
    }
    if (cudaStreamCreateWithFlags(&bs.master, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&bs.fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc(&bs.d_passes, sizeof(unsigned) * n) != cudaSuccess ||
        cudaMalloc(&bs.d_stamp, sizeof(unsigned long long) * (n + 1)) != cudaSuccess ||
        cudaMallocHost(&bs.h_done, sizeof(int) * n) != cudaSuccess) {
        cudaGetLastError();
        return set_error(QCU_ERR_ALLOC, "batch: stream or buffer allocation failed");
    }
    QCUB_CUDA_CHECK(cudaMemsetAsync(bs.d_passes, 0, sizeof(unsigned) * n, bs.master));
    QCUB_CUDA_CHECK(cudaMemsetAsync(bs.d_stamp, 0, sizeof(unsigned long long) * (n + 1), bs.master));
    if ((rc = autotune(bs.sys, o, bs.master))) return rc;
    for (int i = 0; i < n; ++i) {
        System& s = *bs.sys[i];
        s.solve = std::make_unique<SchurSolve>(*s.c, mixed);
        if ((rc = s.solve->begin(s.c->mrhs_out.ptr, s.c->mrhs_in.ptr, sys[i].max_iteration, sys[i].tol)))
            return set_error(rc, "system %d: %s", i, last_message());
    }
    // the graph runs on the master stream: the set-up work of every system must be finished
    for (int i = 0; i < n; ++i) QCUB_CUDA_CHECK(cudaStreamSynchronize(bs.sys[i]->c->stream));
    QCUB_CUDA_CHECK(cudaStreamSynchronize(bs.master));

    const bool host_loop = (flags & QCU_BATCH_HOST_LOOP) != 0;
    if ((rc = host_loop ? capture_host_loop(bs, interval) : capture_device_loop(bs, interval))) return rc;

    std::vector<double> host_latency(n, 0.0);
    if (!host_loop) {
        batch_stamp_kernel<<<1, 1, 0, bs.master>>>(bs.d_stamp + n);
        QCUB_CHECK_LAUNCH();
        QCUB_CUDA_CHECK(cudaGraphLaunch(bs.exec, bs.master));
        QCUB_CUDA_CHECK(cudaStreamSynchronize(bs.master));
    } else {
        int max_launches = 2;
        for (int i = 0; i < n; ++i)
            max_launches = std::max(max_launches, (sys[i].max_iteration + interval - 1) / interval + 2);
        const auto t0 = std::chrono::steady_clock::now();
        int remaining = n;
        for (int l = 0; l < max_launches && remaining > 0; ++l) {
            QCUB_CUDA_CHECK(cudaGraphLaunch(bs.exec, bs.master));
            for (int i = 0; i < n; ++i)
                QCUB_CUDA_CHECK(cudaMemcpyAsync(bs.h_done + i, &bs.sys[i]->solve->device_scalars()->done, sizeof(int),
                                                cudaMemcpyDeviceToHost, bs.master));
            QCUB_CUDA_CHECK(cudaStreamSynchronize(bs.master));
            const double now = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            remaining = 0;
            for (int i = 0; i < n; ++i) {
                if (bs.h_done[i] && host_latency[i] == 0.0) host_latency[i] = now;
                if (!bs.h_done[i]) ++remaining;
            }
        }
    }
    unsigned long long stamps[kMaxBatch + 1] = {};
    if (!host_loop)
        QCUB_CUDA_CHECK(cudaMemcpy(stamps, bs.d_stamp, sizeof(unsigned long long) * (n + 1), cudaMemcpyDeviceToHost));

    int worst = QCU_SUCCESS;
    for (int i = 0; i < n; ++i) {
        System& s = *bs.sys[i];
        Context& c = *s.c;
        c.stats = QcuSolveStats{};
        const int r = s.solve->end();
        if (r != QCU_SUCCESS && r != QCU_ERR_NOT_CONVERGED && r != QCU_ERR_BREAKDOWN) return r;
        if ((rc = move_fields(c, sys[i].x, c.mrhs_out.ptr, false))) return rc;
        sys[i].iterations = c.stats.iterations;
        sys[i].reliable_updates = c.stats.reliable_updates;
        sys[i].status = c.stats.status;
        double worst_res = 0.0;
        for (int j = 0; j < c.m; ++j) worst_res = std::max(worst_res, c.stats.true_residual[j]);
        sys[i].true_residual_max = worst_res;
        sys[i].latency_seconds = host_loop ? host_latency[i]
                                           : (stamps[i] > stamps[n] ? (double)(stamps[i] - stamps[n]) * 1e-9 : 0.0);
        if (c.stats.status != QCU_SUCCESS && worst == QCU_SUCCESS) worst = c.stats.status;
    }
    for (int i = 0; i < n; ++i) QCUB_CUDA_CHECK(cudaStreamSynchronize(bs.sys[i]->c->stream));
    if (worst != QCU_SUCCESS) return set_error(worst, "at least one system of the batch did not converge");
    return QCU_SUCCESS;
}

}  // namespace
}  // namespace qcub

using namespace qcub;

extern "C" int qcuInvertBatch(QcuBatchSystem* systems, int n_systems, const QcuSolverOptions* opts, int flags) {
    clear_error();
    return invert_batch(systems, n_systems, opts, flags);
}

extern "C" int qcuBatchRelease(void) {
    clear_error();
    std::vector<Context*> all;
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        all.swap(g_cache);
    }
    for (Context* c : all) context_destroy(c);
    return QCU_SUCCESS;
}
