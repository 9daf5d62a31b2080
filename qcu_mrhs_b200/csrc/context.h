// context.h -- the host object behind the qcu.h entry points (counterpart of the
// reference class qcu::Qcu, include/qcu_interface.h:12-113).
#pragma once

#include <utility>
#include <vector>

#include "blas.h"
#include "common.cuh"
#include "workspace.h"

namespace qcub {

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

    int64_t half_len() const { return g.vh * 4 * nc; }               // complex per RHS per parity
    size_t half_bytes(int prec) const { return (size_t)half_len() * m * 2 * prec_bytes(prec); }
    int64_t gauge_len() const { return 8 * g.vh * nc * nc; }         // complex numbers

    // gauge in `prec`, created from the FP64 master on first use
    int gauge_in(int prec, const void** out);
};

// Solvers (solver.cu).  b, x: gathered full-lattice fields in FP64 ([2][Vh][4][nc][m]).
int solve_fused(Context& c, void* x, const void* b, int max_iter, double tol);
int solve_mixed(Context& c, void* x, const void* b, int max_iter, double tol);

}  // namespace qcub
