// context.h -- the host object behind the qcu.h entry points (counterpart of the
// reference class qcu::Qcu, include/qcu_interface.h:12-113).
#pragma once

#include <utility>
#include <vector>

#include "blas.h"
#include "common.cuh"
#include "workspace.h"

namespace qcub {

struct Precond;

// Device buffer owned by the context.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    int ensure(size_t nbytes);   // (re)allocate to at least nbytes
    void release();
    ~DevBuf() { release(); }
};

struct Context {
    Geom g{};
    int nc = 3;
    int m = 1;
    int in_prec = QCU_PRECISION_DOUBLE;      // precision of caller fields
    int dslash_prec = QCU_PRECISION_DOUBLE;  // precision of start_dslash / mat_Qcu
    double mass = 0.0;
    double kappa = 0.125;
    bool dslash_ready = false;
    bool gauge_loaded = false;

    // gauge copies by precision code (index 0..4); the FP64 copy is the master
    DevBuf gauge[5];
    bool gauge_valid[5] = {false, false, false, false, false};
    // per-site tables of the tensor-core hop (hop_tables.cu): neighbour table of the
    // lattice, and hop-link arrays by precision with the t-boundary sign they were built for
    DevBuf nbr;
    bool nbr_valid = false;
    DevBuf links[5];
    bool links_valid[5] = {false, false, false, false, false};
    double links_tsign[5] = {0, 0, 0, 0, 0};

    std::vector<std::pair<void*, void*>> queue;   // (out, in) pairs, reference order

    QcuSolverOptions opts{};
    QcuSolveStats stats{};

    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t ev_in = nullptr;     // orders the context stream after the caller's legacy stream
    Scratch ws;

    // gathered field buffers (full lattice: even half then odd half)
    DevBuf mrhs_in, mrhs_out;
    // solver workspace
    DevBuf sv[16];
    DevBuf scalars;           // BicgScalars (device)
    BicgScalars* host_sc = nullptr;   // pinned mirror
    Precond* precond = nullptr;       // learned preconditioner (not owned), QCU_SOLVER_PRECOND
    // executable graph of the last Schur solve's iteration block, updated in place from
    // each new capture (owned)
    cudaGraphExec_t iter_exec = nullptr;

    int64_t half_len() const { return g.vh * 4 * nc; }               // complex per RHS per parity
    size_t half_bytes(int prec) const { return (size_t)half_len() * m * 2 * prec_bytes(prec); }
    int64_t gauge_len() const { return 8 * g.vh * nc * nc; }         // complex numbers

    // gauge in `prec`, created from the FP64 master on first use
    int gauge_in(int prec, const void** out);
    // neighbour table and hop-link array in `prec` for t-boundary sign t_sign, built on
    // first use (outside graph capture)
    int hop_tables(int prec, double t_sign, const void** links_out, const uint32_t** nbr_out);
};

// One Schur BiCGStab solve split into phases, so that several solves can share one
// captured CUDA graph (solver.cu).  b, x: gathered full-lattice fields
// ([2][Vh][4][nc][m], even half first) in the context's input precision (FP64 for
// the mixed solver).
//   begin()             set-up on c.stream: scalars, b', r0 = r = p = b' (synchronises once)
//   enqueue_iteration() one BiCGStab iteration on c.stream, no host synchronisation, so
//                       it may be captured; every kernel returns at once after `done`
//   end()               x_e reconstruction, statistics, FP64 true residual
class SchurSolve {
  public:
    SchurSolve(Context& c, bool mixed) : c_(c), mixed_(mixed) {}
    int begin(void* x, const void* b, int max_iter, double tol);
    int enqueue_iteration();
    int end();
    BicgScalars* device_scalars() const { return dsc_; }

  private:
    int begin_fused(int max_iter, double tol);
    int begin_mixed(int max_iter, double tol);
    Context& c_;
    bool mixed_;
    int P_ = 0, S_ = 0;                 // FP64/FP32 solve precision; sloppy precision
    const void* g_ = nullptr;           // gauge in P_
    const void* gs_ = nullptr;          // gauge in S_ (mixed)
    const void* links_s_ = nullptr;     // per-site tables of the sloppy hop (or null)
    const uint32_t* nbr_s_ = nullptr;
    char* x_ = nullptr;
    const char* b_ = nullptr;
    void* v_[11] = {};
    double2* slots_ = nullptr;
    BicgScalars* dsc_ = nullptr;
    BicgStepArgs a_{};
};

// Whole solves (solver.cu): begin, iterations in graphs of check_interval, end.
int solve_fused(Context& c, void* x, const void* b, int max_iter, double tol);
int solve_mixed(Context& c, void* x, const void* b, int max_iter, double tol);
int solve_cgnr(Context& c, void* x, const void* b, int max_iter, double tol);

// Context life cycle (api.cu), shared by the qcu.h object and the batched solver.
int context_init(Context* c, const int L[4], int n_color, int m_rhs, int in_prec, int dslash_prec);
void context_destroy(Context* c);
// Copy (and cast) a caller gauge field into the context's FP64 master on c->stream.
int context_load_gauge(Context* c, const void* gauge, int prec);

}  // namespace qcub
