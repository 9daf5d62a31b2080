// api.cu -- the qcu.h C interface (reference include/qcu.h, src/interface.cu) and the
// qcu_b200.h extensions, over one process-wide context (the reference keeps a global
// qcu::Qcu*, src/interface.cu:12).  Calls are serialised by a mutex and run on the
// context's own stream; each qcu.h entry point synchronises before returning, as the
// reference does (src/qcu_interface.cu:131,168,359).
#include <mutex>
#include <string>

#include "../../include/qcu.h"
#include "blas.h"
#include "context.h"
#include "dslash.h"
#include "layout.h"
#include "precond.h"

namespace qcub {

int last_status();
int hop_kind();
void set_hop_kind(int k);
int* device_error_flag();
bool hop_mmal_supported(int nc, int m, int prec);
int hop_mmal_launch(const HopParams& p, int nc, int prec, bool dagger, int epi, bool staged, cudaStream_t st);
const char* last_message();

int DevBuf::ensure(size_t nbytes) {
    if (bytes >= nbytes && ptr) return QCU_SUCCESS;
    release();
    const cudaError_t e = cudaMalloc(&ptr, nbytes);
    if (e != cudaSuccess) {
        ptr = nullptr;
        cudaGetLastError();
        return set_error(QCU_ERR_ALLOC, "cudaMalloc(%zu bytes): %s", nbytes, cudaGetErrorString(e));
    }
    bytes = nbytes;
    return QCU_SUCCESS;
}

void DevBuf::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

int Context::gauge_in(int prec, const void** out) {
    if (!gauge_loaded) return set_error(QCU_ERR_STATE, "gauge field not loaded (loadQcuGauge)");
    if (prec < 0 || prec > 4 || prec == QCU_PRECISION_UNDEFINED)
        return set_error(QCU_ERR_INVALID, "precision %d", prec);
    if (!gauge_valid[prec]) {
        int rc = gauge[prec].ensure((size_t)gauge_len() * 2 * prec_bytes(prec));
        if (rc) return rc;
        rc = cast_complex(gauge[prec].ptr, prec, gauge[QCU_PRECISION_DOUBLE].ptr, QCU_PRECISION_DOUBLE,
                          gauge_len(), stream);
        if (rc) return rc;
        gauge_valid[prec] = true;
    }
    *out = gauge[prec].ptr;
    return QCU_SUCCESS;
}

int Context::hop_tables(int prec, double t_sign, const void** links_out, const uint32_t** nbr_out) {
    const void* gp = nullptr;
    int rc = gauge_in(prec, &gp);
    if (rc) return rc;
    if (!nbr_valid) {
        if ((rc = nbr.ensure(neighbour_table_bytes(g)))) return rc;
        if ((rc = build_neighbour_table(static_cast<uint32_t*>(nbr.ptr), nbr.bytes, g, stream))) return rc;
        nbr_valid = true;
    }
    if (!links_valid[prec] || links_tsign[prec] != t_sign) {
        // both output parities: 2 x Vh x 8 links, twice the gauge field
        if ((rc = links[prec].ensure(hop_links_bytes(g, nc, prec)))) return rc;
        if ((rc = build_hop_links(links[prec].ptr, links[prec].bytes, gp, static_cast<const uint32_t*>(nbr.ptr), g, nc,
                                  prec, t_sign, stream)))
            return rc;
        links_valid[prec] = true;
        links_tsign[prec] = t_sign;
    }
    *links_out = links[prec].ptr;
    *nbr_out = static_cast<const uint32_t*>(nbr.ptr);
    return QCU_SUCCESS;
}

static std::mutex g_api;
static Context* g_ctx = nullptr;

static void default_options(QcuSolverOptions* o) {
    o->solver = QCU_SOLVER_FUSED;
    o->sloppy_precision = QCU_PRECISION_BF16;
    o->stop_true_residual = 0;
    o->reliable_delta = 0.1;
    o->t_boundary = 1.0;
    o->check_interval = 8;
    o->freeze_converged = 0;
    o->max_restarts = 0;
    o->reliable_quorum = 0.0;
}

void context_destroy(Context* c) {
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->iter_exec) cudaGraphExecDestroy(c->iter_exec);
    scratch_free(&c->ws);
    if (c->host_sc) cudaFreeHost(c->host_sc);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->ev_in) cudaEventDestroy(c->ev_in);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;   // DevBuf destructors free the buffers
}

// Validate the parameters and create the stream, events, scratch and scalars of a new
// context (c is freshly constructed; on failure the caller destroys it).
int context_init(Context* c, const int L[4], int n_color, int m_rhs, int in_prec, int dslash_prec) {
    if (L[0] < 2 || L[0] % 2 || L[1] < 1 || L[2] < 1 || L[3] < 1)
        return set_error(QCU_ERR_INVALID, "lattice %dx%dx%dx%d (Lx must be even)", L[0], L[1], L[2], L[3]);
    if (n_color < 2 || n_color > kMaxColor)
        return set_error(QCU_ERR_UNSUPPORTED, "n_color=%d (supported 2..%d)", n_color, kMaxColor);
    if (m_rhs < 1 || m_rhs > kMaxRhs) return set_error(QCU_ERR_INVALID, "m_rhs=%d (1..%d)", m_rhs, kMaxRhs);
    if (!prec_valid(in_prec)) return set_error(QCU_ERR_INVALID, "input precision %d", in_prec);
    if (!prec_valid(dslash_prec)) return set_error(QCU_ERR_INVALID, "dslash precision %d", dslash_prec);
    c->g = make_geom(L);
    c->nc = n_color;
    c->m = m_rhs;
    c->in_prec = in_prec;
    c->dslash_prec = dslash_prec;
    default_options(&c->opts);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_in, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return set_error(QCU_ERR_CUDA, "stream/event creation failed");
    }
    int rc = scratch_alloc(&c->ws);
    if (!rc) rc = c->scalars.ensure(sizeof(BicgScalars));
    if (!rc && cudaMallocHost(&c->host_sc, sizeof(BicgScalars)) != cudaSuccess) {
        cudaGetLastError();
        rc = set_error(QCU_ERR_ALLOC, "pinned host allocation failed");
    }
    if (!rc) rc = hop16_pairs_prepare();   // before any solve is captured into a graph
    if (!rc) rc = hop_mmal_prepare();
    return rc;
}

int context_load_gauge(Context* c, const void* gauge, int prec) {
    if (!gauge) return set_error(QCU_ERR_INVALID, "null gauge pointer");
    if (!prec_valid(prec)) return set_error(QCU_ERR_INVALID, "gauge precision %d", prec);
    const int D = QCU_PRECISION_DOUBLE;
    int rc;
    if ((rc = c->gauge[D].ensure((size_t)c->gauge_len() * 16))) return rc;
    if ((rc = cast_complex(c->gauge[D].ptr, D, gauge, prec, c->gauge_len(), c->stream))) return rc;
    for (int i = 0; i < 5; ++i) c->gauge_valid[i] = c->links_valid[i] = false;
    c->gauge_valid[D] = true;
    c->gauge_loaded = true;
    return QCU_SUCCESS;
}

static int require_ctx() {
    if (!g_ctx) return set_error(QCU_ERR_STATE, "Qcu is not initialized (initGridSize)");
    return QCU_SUCCESS;
}

// Work the caller queued on the legacy default stream (where the reference runs) is
// finished before the context's stream reads the caller's buffers.
static int order_after_caller(Context& c) {
    QCUB_CUDA_CHECK(cudaEventRecord(c.ev_in, 0));
    QCUB_CUDA_CHECK(cudaStreamWaitEvent(c.stream, c.ev_in, 0));
    return QCU_SUCCESS;
}

static int require_queue(Context& c) {
    if ((int)c.queue.size() != c.m)
        return set_error(QCU_ERR_STATE, "fermion queue holds %d of %d pairs", (int)c.queue.size(), c.m);
    return QCU_SUCCESS;
}

static int require_dslash(Context& c) {
    if (!c.dslash_ready) return set_error(QCU_ERR_STATE, "Dslash is not initialized (getDslash)");
    if (!c.gauge_loaded) return set_error(QCU_ERR_STATE, "gauge field not loaded (loadQcuGauge)");
    return QCU_SUCCESS;
}

// ---------------- qcu.h ----------------

static int init_impl(QcuGrid* grid, QcuParam* param, int n_color, int m_rhs, int in_prec, int dslash_prec) {
    if (!grid || !param) return set_error(QCU_ERR_INVALID, "null grid or param");
    for (int i = 0; i < 4; ++i)
        if (grid->grid_size[i] != 1)
            return set_error(QCU_ERR_UNSUPPORTED, "process grid %d,%d,%d,%d: one GPU needs 1,1,1,1",
                             grid->grid_size[0], grid->grid_size[1], grid->grid_size[2], grid->grid_size[3]);
    Context* c = new Context();
    const int rc = context_init(c, param->lattice_size, n_color, m_rhs, in_prec, dslash_prec);
    if (rc) {
        context_destroy(c);
        return rc;
    }
    context_destroy(g_ctx);
    g_ctx = c;
    return QCU_SUCCESS;
}

static int load_gauge_impl(void* gauge, int prec) {
    int rc = require_ctx();
    if (rc) return rc;
    Context& c = *g_ctx;
    if (!gauge) return set_error(QCU_ERR_INVALID, "null gauge pointer");
    if ((rc = order_after_caller(c))) return rc;
    if ((rc = context_load_gauge(&c, gauge, prec))) return rc;
    QCUB_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    return QCU_SUCCESS;
}

static int get_dslash_impl(int type, double mass) {
    int rc = require_ctx();
    if (rc) return rc;
    if (type != QCU_DSLASH_WILSON) return set_error(QCU_ERR_UNSUPPORTED, "dslash type %d (Wilson = 0)", type);
    g_ctx->mass = mass;
    g_ctx->kappa = 1.0 / (2.0 * (4.0 + mass));
    g_ctx->dslash_ready = true;
    return QCU_SUCCESS;
}

static int push_impl(void* out, void* in) {
    int rc = require_ctx();
    if (rc) return rc;
    if ((int)g_ctx->queue.size() >= g_ctx->m) return set_error(QCU_ERR_STATE, "Fermion queue is full");
    if (!out || !in) return set_error(QCU_ERR_INVALID, "null fermion pointer");
    g_ctx->queue.emplace_back(out, in);
    return QCU_SUCCESS;
}

static void clear_queue() {
    if (g_ctx) g_ctx->queue.clear();
}

// out[parity] = D in[1 - parity] on half-lattice per-RHS fields, in dslash precision
static int start_dslash_impl(int parity, int dagger) {
    int rc = require_ctx();
    if (rc) return rc;
    Context& c = *g_ctx;
    if ((rc = require_dslash(c)) || (rc = require_queue(c))) return rc;
    if (parity != 0 && parity != 1) return set_error(QCU_ERR_INVALID, "parity %d", parity);
    if ((rc = order_after_caller(c))) return rc;
    const int Pd = c.dslash_prec;
    const void* gauge = nullptr;
    if ((rc = c.gauge_in(Pd, &gauge))) return rc;
    const size_t hb = c.half_bytes(Pd);
    if ((rc = c.mrhs_in.ensure(hb)) || (rc = c.mrhs_out.ensure(hb))) return rc;
    void* ins[kMaxRhs];
    void* outs[kMaxRhs];
    for (int j = 0; j < c.m; ++j) {
        outs[j] = c.queue[j].first;
        ins[j] = c.queue[j].second;
    }
    if ((rc = gather_mrhs(c.mrhs_in.ptr, Pd, ins, c.in_prec, c.g.vh, c.nc, c.m, c.stream))) return rc;
    const void* links = nullptr;
    const uint32_t* nbr = nullptr;
    if (hop_reads_tables(c.nc, c.m, Pd) && (rc = c.hop_tables(Pd, c.opts.t_boundary, &links, &nbr))) return rc;
    HopParams p{};
    p.links = links;
    p.nbr = nbr;
    p.out = c.mrhs_out.ptr;
    p.in = c.mrhs_in.ptr;
    p.gauge = gauge;
    p.g = c.g;
    p.m = c.m;
    p.parity = parity;
    p.t_sign = c.opts.t_boundary;
    if ((rc = hop_launch(p, c.nc, Pd, dagger != 0, EPI_PLAIN, c.stream))) return rc;
    if ((rc = scatter_mrhs(outs, c.in_prec, c.mrhs_out.ptr, Pd, c.g.vh, c.nc, c.m, c.stream))) return rc;
    QCUB_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    return QCU_SUCCESS;
}

// out = in - kappa D in on full-lattice per-RHS fields (reference src/qcu_interface.cu:174-256)
static int mat_impl(int dagger) {
    int rc = require_ctx();
    if (rc) return rc;
    Context& c = *g_ctx;
    if ((rc = require_dslash(c)) || (rc = require_queue(c))) return rc;
    if ((rc = order_after_caller(c))) return rc;
    const int Pd = c.dslash_prec;
    const void* gauge = nullptr;
    if ((rc = c.gauge_in(Pd, &gauge))) return rc;
    const size_t hb = c.half_bytes(Pd);
    if ((rc = c.mrhs_in.ensure(2 * hb)) || (rc = c.mrhs_out.ensure(2 * hb))) return rc;
    const size_t half_ext = (size_t)c.g.vh * 4 * c.nc * 2 * prec_bytes(c.in_prec);  // one parity, one RHS
    void* ins[2][kMaxRhs];
    void* outs[2][kMaxRhs];
    for (int j = 0; j < c.m; ++j)
        for (int par = 0; par < 2; ++par) {
            ins[par][j] = static_cast<char*>(c.queue[j].second) + par * half_ext;
            outs[par][j] = static_cast<char*>(c.queue[j].first) + par * half_ext;
        }
    char* gin = static_cast<char*>(c.mrhs_in.ptr);
    char* gout = static_cast<char*>(c.mrhs_out.ptr);
    for (int par = 0; par < 2; ++par)
        if ((rc = gather_mrhs(gin + par * hb, Pd, ins[par], c.in_prec, c.g.vh, c.nc, c.m, c.stream))) return rc;
    const void* links = nullptr;
    const uint32_t* nbr = nullptr;
    if (hop_reads_tables(c.nc, c.m, Pd) && (rc = c.hop_tables(Pd, c.opts.t_boundary, &links, &nbr))) return rc;
    for (int par = 0; par < 2; ++par) {
        HopParams p{};
        p.links = links;
        p.nbr = nbr;
        p.out = gout + par * hb;
        p.in = gin + (1 - par) * hb;
        p.x = gin + par * hb;
        p.a = -c.kappa;
        p.gauge = gauge;
        p.g = c.g;
        p.m = c.m;
        p.parity = par;
        p.t_sign = c.opts.t_boundary;
        if ((rc = hop_launch(p, c.nc, Pd, dagger != 0, EPI_XPAY, c.stream))) return rc;
    }
    for (int par = 0; par < 2; ++par)
        if ((rc = scatter_mrhs(outs[par], c.in_prec, gout + par * hb, Pd, c.g.vh, c.nc, c.m, c.stream))) return rc;
    QCUB_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    return QCU_SUCCESS;
}

static int invert_impl(int max_iter, double tol) {
    int rc = require_ctx();
    if (rc) return rc;
    Context& c = *g_ctx;
    if ((rc = require_dslash(c)) || (rc = require_queue(c))) return rc;
    if (!(tol > 0)) return set_error(QCU_ERR_INVALID, "tolerance %g", tol);
    if ((rc = order_after_caller(c))) return rc;
    const bool mixed = c.opts.solver == QCU_SOLVER_MIXED;
    const int P = c.in_prec;
    if (!mixed && P != QCU_PRECISION_DOUBLE && P != QCU_PRECISION_SINGLE)
        return set_error(QCU_ERR_UNSUPPORTED, "output precision must be float or double");
    const size_t hb = c.half_bytes(P);
    if ((rc = c.mrhs_in.ensure(2 * hb)) || (rc = c.mrhs_out.ensure(2 * hb))) return rc;
    const size_t half_ext = (size_t)c.g.vh * 4 * c.nc * 2 * prec_bytes(P);
    void* ins[2][kMaxRhs];
    void* outs[2][kMaxRhs];
    for (int j = 0; j < c.m; ++j)
        for (int par = 0; par < 2; ++par) {
            ins[par][j] = static_cast<char*>(c.queue[j].second) + par * half_ext;
            outs[par][j] = static_cast<char*>(c.queue[j].first) + par * half_ext;
        }
    char* b = static_cast<char*>(c.mrhs_in.ptr);
    char* x = static_cast<char*>(c.mrhs_out.ptr);
    for (int par = 0; par < 2; ++par)
        if ((rc = gather_mrhs(b + par * hb, P, ins[par], P, c.g.vh, c.nc, c.m, c.stream))) return rc;
    c.stats = QcuSolveStats{};
    if (c.opts.solver == QCU_SOLVER_PRECOND)
        rc = solve_precond(c, c.precond, x, b, max_iter, tol);
    else if (c.opts.solver == QCU_SOLVER_CGNR)
        rc = solve_cgnr(c, x, b, max_iter, tol);
    else
        rc = mixed ? solve_mixed(c, x, b, max_iter, tol) : solve_fused(c, x, b, max_iter, tol);
    const int solve_rc = rc;
    const std::string solve_msg = last_message();   // a copy: set_error below rewrites the buffer
    if (rc != QCU_SUCCESS && rc != QCU_ERR_NOT_CONVERGED && rc != QCU_ERR_BREAKDOWN) return rc;
    // write the solution (also the last iterate when not converged)
    for (int par = 0; par < 2; ++par)
        if ((rc = scatter_mrhs(outs[par], P, x + par * hb, P, c.g.vh, c.nc, c.m, c.stream))) return rc;
    QCUB_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    if (solve_rc != QCU_SUCCESS) return set_error(solve_rc, "%s", solve_msg.c_str());
    return QCU_SUCCESS;
}

static int gauge_eo_impl(void* dst, void* src, int prec, int to_eo) {
    int rc = require_ctx();
    if (rc) return rc;
    Context& c = *g_ctx;
    if (!dst || !src) return set_error(QCU_ERR_INVALID, "null gauge pointer");
    if ((rc = order_after_caller(c))) return rc;
    if ((rc = gauge_reorder(dst, src, c.g.L, c.nc, prec, to_eo, c.stream))) return rc;
    QCUB_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    return QCU_SUCCESS;
}

}  // namespace qcub

using namespace qcub;

#define QCUB_API_BEGIN               \
    std::lock_guard<std::mutex> lk(g_api); \
    clear_error();

extern "C" {

void initGridSize(QcuGrid* grid, QcuParam* param, int n_color, int m_rhs, int inputFloatPrecision,
                  int dslashFloatPrecision) {
    QCUB_API_BEGIN
    init_impl(grid, param, n_color, m_rhs, inputFloatPrecision, dslashFloatPrecision);
}

void pushBackFermions(void* fermionOut, void* fermionIn) {
    QCUB_API_BEGIN
    push_impl(fermionOut, fermionIn);
}

void loadQcuGauge(void* gauge, int floatPrecision) {
    QCUB_API_BEGIN
    load_gauge_impl(gauge, floatPrecision);
}

void getDslash(int dslashType, double mass) {
    QCUB_API_BEGIN
    get_dslash_impl(dslashType, mass);
}

void start_dslash(int parity, int daggerFlag) {
    QCUB_API_BEGIN
    start_dslash_impl(parity, daggerFlag);
    clear_queue();
}

void mat_Qcu(int daggerFlag) {
    QCUB_API_BEGIN
    mat_impl(daggerFlag);
    clear_queue();
}

void qcuInvert(int max_iteration, double p_max_prec) {
    QCUB_API_BEGIN
    invert_impl(max_iteration, p_max_prec);
    clear_queue();
}

void finalizeQcu() {
    QCUB_API_BEGIN
    context_destroy(g_ctx);
    g_ctx = nullptr;
}

void gauge_eo_precondition(void* prec_gauge, void* non_prec_gauge, int precision) {
    QCUB_API_BEGIN
    gauge_eo_impl(prec_gauge, non_prec_gauge, precision, 1);
}

void gauge_reverse_eo_precondition(void* non_prec_gauge, void* prec_gauge, int precision) {
    QCUB_API_BEGIN
    gauge_eo_impl(non_prec_gauge, prec_gauge, precision, 0);
}

void read_gauge_from_file(void* gauge, const char* file_path_prefix) {
    QCUB_API_BEGIN
    (void)gauge;
    (void)file_path_prefix;
    set_error(QCU_ERR_UNSUPPORTED,
              "read_gauge_from_file: the gauge file format is defined outside the reference tree");
}

// ---------------- qcu_b200.h ----------------

int qcuGetLastStatus(void) { return last_status(); }
const char* qcuGetLastError(void) { return last_message(); }

void qcuGetDefaultSolverOptions(QcuSolverOptions* opts) {
    if (opts) default_options(opts);
}

int qcuSetSolverOptions(const QcuSolverOptions* opts) {
    QCUB_API_BEGIN
    int rc = require_ctx();
    if (rc) return rc;
    if (!opts) return set_error(QCU_ERR_INVALID, "null options");
    if (opts->solver < QCU_SOLVER_REFERENCE || opts->solver > QCU_SOLVER_CGNR)
        return set_error(QCU_ERR_INVALID, "solver %d", opts->solver);
    if (opts->t_boundary != 1.0 && opts->t_boundary != -1.0)
        return set_error(QCU_ERR_INVALID, "t_boundary must be +1 or -1");
    g_ctx->opts = *opts;
    return QCU_SUCCESS;
}

int qcuSetPreconditioner(void* handle) {
    QCUB_API_BEGIN
    int rc = require_ctx();
    if (rc) return rc;
    Precond* P = static_cast<Precond*>(handle);
    if (P) {
        for (int i = 0; i < 4; ++i)
            if (P->g.L[i] != g_ctx->g.L[i]) return set_error(QCU_ERR_INVALID, "preconditioner lattice differs");
        if (P->nc != g_ctx->nc || P->m != g_ctx->m)
            return set_error(QCU_ERR_INVALID, "preconditioner n_color / m_rhs differ from the context");
    }
    g_ctx->precond = P;
    return QCU_SUCCESS;
}

int qcuGetSolveStats(QcuSolveStats* stats) {
    QCUB_API_BEGIN
    int rc = require_ctx();
    if (rc) return rc;
    if (!stats) return set_error(QCU_ERR_INVALID, "null stats");
    *stats = g_ctx->stats;
    return QCU_SUCCESS;
}

static int hop_common(void* out, const void* in, const void* gauge, const void* x, double a,
                      const int L[4], int n_color, int m_rhs, int parity, int dagger, double t_sign,
                      int precision, void* stream, int epi) {
    if (!out || !in || !gauge || !L) return set_error(QCU_ERR_INVALID, "null pointer");
    if (epi == EPI_XPAY && !x) return set_error(QCU_ERR_INVALID, "null x");
    if (parity != 0 && parity != 1) return set_error(QCU_ERR_INVALID, "parity %d", parity);
    HopParams p{};
    p.out = out;
    p.in = in;
    p.gauge = gauge;
    p.x = x;
    p.a = a;
    p.g = make_geom(L);
    p.m = m_rhs;
    p.parity = parity;
    p.t_sign = t_sign;
    return hop_launch(p, n_color, precision, dagger != 0, epi, static_cast<cudaStream_t>(stream));
}

int qcuDslashMrhs(void* out, const void* in, const void* gauge, const int L[4], int n_color, int m_rhs,
                  int parity, int dagger, double t_sign, int precision, void* stream) {
    clear_error();
    return hop_common(out, in, gauge, nullptr, 0.0, L, n_color, m_rhs, parity, dagger, t_sign, precision,
                      stream, EPI_PLAIN);
}

int qcuDslashMrhsXpay(void* out, const void* in, const void* gauge, const void* x, double a,
                      const int L[4], int n_color, int m_rhs, int parity, int dagger, double t_sign,
                      int precision, void* stream) {
    clear_error();
    return hop_common(out, in, gauge, x, a, L, n_color, m_rhs, parity, dagger, t_sign, precision, stream,
                      EPI_XPAY);
}

// the context's hop (caller holds the API lock); epi selects the fused epilogue (x, r0 and a
// are its operands, red the [nval][m] double2 output of its reduction or null for scratch)
static int context_hop(void* out, const void* in, int parity, int dagger, int precision, const int* active,
                       void* stream, int epi = EPI_PLAIN, const void* x = nullptr, const void* r0 = nullptr,
                       double a = 0.0, void* red = nullptr) {
    int rc = require_ctx();
    if (rc) return rc;
    Context& c = *g_ctx;
    if ((rc = require_dslash(c))) return rc;
    if (!out || !in) return set_error(QCU_ERR_INVALID, "null pointer");
    if (parity != 0 && parity != 1) return set_error(QCU_ERR_INVALID, "parity %d", parity);
    const void* gauge = nullptr;
    if ((rc = c.gauge_in(precision, &gauge))) return rc;
    const void* links = nullptr;
    const uint32_t* nbr = nullptr;
    if (hop_reads_tables(c.nc, c.m, precision) &&
        (rc = c.hop_tables(precision, c.opts.t_boundary, &links, &nbr)))
        return rc;
    // the gauge copy and tables were made on the context's stream: order the caller's after it
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    QCUB_CUDA_CHECK(cudaEventRecord(c.ev_in, c.stream));
    QCUB_CUDA_CHECK(cudaStreamWaitEvent(st, c.ev_in, 0));
    HopParams p{};
    p.out = out;
    p.in = in;
    p.gauge = gauge;
    p.links = links;
    p.nbr = nbr;
    p.g = c.g;
    p.m = c.m;
    p.parity = parity;
    p.t_sign = c.opts.t_boundary;
    p.active = active;
    p.x = x;
    p.r0 = r0;
    p.a = a;
    if (epi == EPI_SCHUR_R0 || epi == EPI_SCHUR_TS || epi == EPI_RESID) {
        // the reduction's scratch is the context's, used on its stream: order the caller's
        // stream after it and the context's stream after this launch
        p.red = RedArgs{c.ws.partials, c.ws.counter, red ? static_cast<double2*>(red) : c.ws.result, nullptr,
                        nullptr, FIN_NONE};
    }
    int rc2 = hop_launch(p, c.nc, precision, dagger != 0, epi, st);
    if (rc2 == QCU_SUCCESS && p.red.partials) {
        QCUB_CUDA_CHECK(cudaEventRecord(c.ev_in, st));
        QCUB_CUDA_CHECK(cudaStreamWaitEvent(c.stream, c.ev_in, 0));
    }
    return rc2;
}

int qcuDslashMrhsContext(void* out, const void* in, int parity, int dagger, int precision, void* stream) {
    QCUB_API_BEGIN
    return context_hop(out, in, parity, dagger, precision, nullptr, stream);
}

int qcuDslashMrhsContextActive(void* out, const void* in, int parity, int dagger, int precision,
                               const int* active, void* stream) {
    QCUB_API_BEGIN
    if (!active) return set_error(QCU_ERR_INVALID, "null activity flags");
    return context_hop(out, in, parity, dagger, precision, active, stream);
}

static_assert(QCU_HOP_FORM_PLAIN == EPI_PLAIN && QCU_HOP_FORM_XPAY == EPI_XPAY &&
                  QCU_HOP_FORM_SCHUR_R0 == EPI_SCHUR_R0 && QCU_HOP_FORM_SCHUR_TS == EPI_SCHUR_TS &&
                  QCU_HOP_FORM_SCHUR == EPI_SCHUR && QCU_HOP_FORM_RESID == EPI_RESID,
              "hop form codes are the epilogue codes");

int qcuDslashMrhsContextForm(void* out, const void* in, const void* x, const void* r0, double a, int form,
                             int parity, int precision, void* red, void* stream) {
    QCUB_API_BEGIN
    if (form < QCU_HOP_FORM_PLAIN || form > QCU_HOP_FORM_RESID)
        return set_error(QCU_ERR_INVALID, "hop form %d", form);
    if (form != QCU_HOP_FORM_PLAIN && !x) return set_error(QCU_ERR_INVALID, "hop form %d needs x", form);
    if ((form == QCU_HOP_FORM_SCHUR_R0 || form == QCU_HOP_FORM_RESID) && !r0)
        return set_error(QCU_ERR_INVALID, "hop form %d needs r0", form);
    return context_hop(out, in, parity, 0, precision, nullptr, stream, form, x, r0, a, red);
}

int qcuSchurMrhs(void* out, const void* in, void* tmp, const void* gauge, double kappa, const int L[4],
                 int n_color, int m_rhs, double t_sign, int precision, void* stream) {
    clear_error();
    if (!tmp) return set_error(QCU_ERR_INVALID, "null tmp");
    int rc = hop_common(tmp, in, gauge, nullptr, 0.0, L, n_color, m_rhs, 0, 0, t_sign, precision, stream,
                        EPI_PLAIN);
    if (rc) return rc;
    HopParams p{};
    p.out = out;
    p.in = tmp;
    p.gauge = gauge;
    p.x = in;
    p.a = kappa * kappa;
    p.g = make_geom(L);
    p.m = m_rhs;
    p.parity = 1;
    p.t_sign = t_sign;
    return hop_launch(p, n_color, precision, false, EPI_SCHUR, static_cast<cudaStream_t>(stream));
}

int qcuGatherMrhs(void* dst, int dst_precision, void* const* src_ptrs, int src_precision, int64_t vh,
                  int n_color, int m_rhs, void* stream) {
    clear_error();
    if (!dst || !src_ptrs) return set_error(QCU_ERR_INVALID, "null pointer");
    return gather_mrhs(dst, dst_precision, src_ptrs, src_precision, vh, n_color, m_rhs,
                       static_cast<cudaStream_t>(stream));
}

int qcuScatterMrhs(void* const* dst_ptrs, int dst_precision, const void* src, int src_precision,
                   int64_t vh, int n_color, int m_rhs, void* stream) {
    clear_error();
    if (!src || !dst_ptrs) return set_error(QCU_ERR_INVALID, "null pointer");
    return scatter_mrhs(dst_ptrs, dst_precision, src, src_precision, vh, n_color, m_rhs,
                        static_cast<cudaStream_t>(stream));
}

int qcuCopyComplexVector(void* dst, int dst_precision, const void* src, int src_precision, int64_t n,
                         void* stream) {
    clear_error();
    if ((!dst || !src) && n > 0) return set_error(QCU_ERR_INVALID, "null pointer");
    return cast_complex(dst, dst_precision, src, src_precision, n, static_cast<cudaStream_t>(stream));
}

int qcuMrhsDotc(void* res, const void* a, const void* b, int64_t len, int m, int precision, void* stream) {
    clear_error();
    int rc = check_mrhs(len, m);
    if (rc) return rc;
    if (!res || !a || !b) return set_error(QCU_ERR_INVALID, "null pointer");
    const Scratch* ws = nullptr;
    if ((rc = device_scratch(&ws))) return rc;
    return mrhs_dotc(static_cast<double2*>(res), a, b, len, m, precision, *ws,
                     static_cast<cudaStream_t>(stream));
}

int qcuMrhsNorm(double* res, const void* a, int64_t len, int m, int precision, void* stream) {
    clear_error();
    int rc = check_mrhs(len, m);
    if (rc) return rc;
    if (!res || !a) return set_error(QCU_ERR_INVALID, "null pointer");
    const Scratch* ws = nullptr;
    if ((rc = device_scratch(&ws))) return rc;
    return mrhs_norm(res, a, len, m, precision, *ws, static_cast<cudaStream_t>(stream));
}

static int axpy_common(int op, void* res, const void* a, const void* x, const void* b, const void* y,
                       const void* c, const void* z, int64_t len, int m, int precision, void* stream) {
    clear_error();
    int rc = check_mrhs(len, m);
    if (rc) return rc;
    if (!res || !a || !x || !y) return set_error(QCU_ERR_INVALID, "null pointer");
    if (op >= OP_AXPBY && !b) return set_error(QCU_ERR_INVALID, "null pointer");
    if (op == OP_AXPBYPCZ && (!c || !z)) return set_error(QCU_ERR_INVALID, "null pointer");
    return mrhs_axpy(op, res, a, x, b, y, c, z, len, m, precision, static_cast<cudaStream_t>(stream));
}

int qcuMrhsXsay(void* res, const void* x, const void* a, const void* y, int64_t len, int m, int precision,
                void* stream) {
    return axpy_common(OP_XSAY, res, a, x, nullptr, y, nullptr, nullptr, len, m, precision, stream);
}

int qcuMrhsXpay(void* res, const void* x, const void* a, const void* y, int64_t len, int m, int precision,
                void* stream) {
    return axpy_common(OP_XPAY, res, a, x, nullptr, y, nullptr, nullptr, len, m, precision, stream);
}

int qcuMrhsAxpby(void* res, const void* a, const void* x, const void* b, const void* y, int64_t len, int m,
                 int precision, void* stream) {
    return axpy_common(OP_AXPBY, res, a, x, b, y, nullptr, nullptr, len, m, precision, stream);
}

int qcuMrhsAxpbypcz(void* res, const void* a, const void* x, const void* b, const void* y, const void* c,
                    const void* z, int64_t len, int m, int precision, void* stream) {
    return axpy_common(OP_AXPBYPCZ, res, a, x, b, y, c, z, len, m, precision, stream);
}

int qcuElementwiseDiv(void* res, const void* x, const void* y, int m, void* stream) {
    clear_error();
    if (!res || !x || !y) return set_error(QCU_ERR_INVALID, "null pointer");
    return elementwise(0, res, x, y, m, 0, 0, static_cast<cudaStream_t>(stream));
}

int qcuElementwiseMul(void* res, const void* x, const void* y, int m, void* stream) {
    clear_error();
    if (!res || !x || !y) return set_error(QCU_ERR_INVALID, "null pointer");
    return elementwise(1, res, x, y, m, 0, 0, static_cast<cudaStream_t>(stream));
}

int qcuElementwiseInit(void* res, double re, double im, int m, void* stream) {
    clear_error();
    if (!res) return set_error(QCU_ERR_INVALID, "null pointer");
    return elementwise(2, res, nullptr, nullptr, m, re, im, static_cast<cudaStream_t>(stream));
}

int qcuGaugeToEO(void* eo, const void* lex, const int L[4], int n_color, int precision, void* stream) {
    clear_error();
    if (!eo || !lex || !L) return set_error(QCU_ERR_INVALID, "null pointer");
    return gauge_reorder(eo, lex, L, n_color, precision, 1, static_cast<cudaStream_t>(stream));
}

int qcuGaugeFromEO(void* lex, const void* eo, const int L[4], int n_color, int precision, void* stream) {
    clear_error();
    if (!eo || !lex || !L) return set_error(QCU_ERR_INVALID, "null pointer");
    return gauge_reorder(lex, eo, L, n_color, precision, 0, static_cast<cudaStream_t>(stream));
}

int qcuFermionToEO(void* eo, const void* lex, const int L[4], int n_color, int precision, void* stream) {
    clear_error();
    if (!eo || !lex || !L) return set_error(QCU_ERR_INVALID, "null pointer");
    if (n_color < 1 || n_color > kMaxColor) return set_error(QCU_ERR_INVALID, "n_color=%d", n_color);
    return fermion_reorder(eo, lex, L, n_color, precision, 1, static_cast<cudaStream_t>(stream));
}

int qcuFermionFromEO(void* lex, const void* eo, const int L[4], int n_color, int precision, void* stream) {
    clear_error();
    if (!eo || !lex || !L) return set_error(QCU_ERR_INVALID, "null pointer");
    if (n_color < 1 || n_color > kMaxColor) return set_error(QCU_ERR_INVALID, "n_color=%d", n_color);
    return fermion_reorder(lex, eo, L, n_color, precision, 0, static_cast<cudaStream_t>(stream));
}

int qcuSiteBlockMrhs(void* dst, const void* src, int64_t vh, int n_color, int m_rhs, int precision,
                     int to_blocked, void* stream) {
    clear_error();
    if (to_blocked != 0 && to_blocked != 1) return set_error(QCU_ERR_INVALID, "to_blocked %d", to_blocked);
    return site_block_reorder(dst, src, vh, n_color, m_rhs, precision, to_blocked, static_cast<cudaStream_t>(stream));
}

int qcuDslashMrhsSiteBlocked(void* out, const void* in, const void* gauge, const int L[4], int n_color, int m_rhs,
                             int parity, int dagger, double t_sign, int precision, void* stream) {
    clear_error();
    if (!out || !in || !gauge || !L) return set_error(QCU_ERR_INVALID, "null pointer");
    if (parity != 0 && parity != 1) return set_error(QCU_ERR_INVALID, "parity %d", parity);
    HopParams p{};
    p.out = out;
    p.in = in;
    p.gauge = gauge;
    p.g = make_geom(L);
    p.m = m_rhs;
    p.parity = parity;
    p.t_sign = t_sign;
    p.blocked = 1;
    return hop_launch(p, n_color, precision, dagger != 0, EPI_PLAIN, static_cast<cudaStream_t>(stream));
}

int qcuSetHopKernel(int kind) {
    clear_error();
    if (kind < QCU_HOP_AUTO || kind > QCU_HOP_MMA_LINK_DIRECT)
        return set_error(QCU_ERR_INVALID, "hop kernel kind %d", kind);
    set_hop_kind(kind);
    return QCU_SUCCESS;
}

int qcuGetHopKernel(void) { return hop_kind(); }

int qcuGetKernelError(int clear) {
    clear_error();
    int* flag = device_error_flag();
    if (!flag) return set_error(QCU_ERR_CUDA, "device error flag unavailable");
    QCUB_CUDA_CHECK(cudaDeviceSynchronize());
    int h = 0;
    QCUB_CUDA_CHECK(cudaMemcpy(&h, flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (clear) QCUB_CUDA_CHECK(cudaMemset(flag, 0, sizeof(int)));
    return h;
}

int qcuHopWaitSelfTest(long long limit_cycles, int* timed_out) {
    QCUB_API_BEGIN
    if (!timed_out || limit_cycles < 1) return set_error(QCU_ERR_INVALID, "qcuHopWaitSelfTest: arguments");
    int rc = require_ctx();
    if (rc) return rc;
    Context& c = *g_ctx;
    if ((rc = require_dslash(c))) return rc;
    const int prec = QCU_PRECISION_HALF;
    if (!hop_mmal_supported(c.nc, c.m, prec) || c.nc > 4 || c.m > 16 || c.m % 4)
        return set_error(QCU_ERR_UNSUPPORTED, "qcuHopWaitSelfTest: the staged hop needs n_color <= 4, m_rhs = 4..16");
    const void* gauge = nullptr;
    const void* links = nullptr;
    const uint32_t* nbr = nullptr;
    if ((rc = c.gauge_in(prec, &gauge))) return rc;
    if ((rc = c.hop_tables(prec, c.opts.t_boundary, &links, &nbr))) return rc;
    int* flag = device_error_flag();
    if (!flag) return set_error(QCU_ERR_CUDA, "device error flag unavailable");
    void* buf = nullptr;
    const size_t hb = c.half_bytes(prec);
    QCUB_CUDA_CHECK(cudaMalloc(&buf, 2 * hb));
    HopParams p{};
    p.out = static_cast<char*>(buf) + hb;
    p.in = buf;
    p.gauge = gauge;
    p.links = links;
    p.nbr = nbr;
    p.g = c.g;
    p.m = c.m;
    p.parity = 0;
    p.t_sign = c.opts.t_boundary;
    p.wait_limit = limit_cycles;
    p.wait_test = 1;
    cudaError_t e = cudaStreamSynchronize(c.stream);
    if (e == cudaSuccess) e = cudaMemset(flag, 0, sizeof(int));
    if (e == cudaSuccess) {
        rc = hop_mmal_launch(p, c.nc, prec, false, EPI_PLAIN, true, c.stream);
        if (rc == QCU_SUCCESS) e = cudaStreamSynchronize(c.stream);
    }
    int h = 0;
    if (rc == QCU_SUCCESS && e == cudaSuccess) e = cudaMemcpy(&h, flag, sizeof(int), cudaMemcpyDeviceToHost);
    if (rc == QCU_SUCCESS && e == cudaSuccess) e = cudaMemset(flag, 0, sizeof(int));
    cudaFree(buf);
    if (rc) return rc;
    if (e != cudaSuccess) return set_error(QCU_ERR_CUDA, "qcuHopWaitSelfTest: %s", cudaGetErrorString(e));
    *timed_out = h != 0;
    return QCU_SUCCESS;
}

int qcuDeviceSynchronize(void) {
    clear_error();
    QCUB_CUDA_CHECK(cudaDeviceSynchronize());
    return QCU_SUCCESS;
}

}  // extern "C"
