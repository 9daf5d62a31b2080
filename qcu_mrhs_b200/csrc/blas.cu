// blas.cu -- host entry points of the multi-RHS BLAS (qcu_b200.h) and launch helpers
// for the fused BiCGStab steps.
#include "blas.h"
#include "blas_impl.cuh"
#include "workspace.h"

namespace qcub {

int check_mrhs(int64_t len, int m) {
    if (m < 1 || m > kMaxRhs) return set_error(QCU_ERR_INVALID, "m_rhs=%d outside [1, %d]", m, kMaxRhs);
    if (len < 0) return set_error(QCU_ERR_INVALID, "negative vector length");
    return QCU_SUCCESS;
}

template <typename S>
static int dotc_t(double2* res, const void* a, const void* b, int64_t len, int m, const Scratch& ws,
                  cudaStream_t st) {
    using S2 = typename St<S>::S2;
    const int block = rhs_block(m);
    auto k = dotc_kernel<S>;
    int grid = resident_grid(k, block, len * m);
    if (grid > ws.max_blocks) grid = ws.max_blocks;
    RedArgs ra{ws.partials, ws.counter, res, nullptr, nullptr, FIN_NONE};
    k<<<grid, block, 0, st>>>(static_cast<const S2*>(a), static_cast<const S2*>(b), len * m, m, ra);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

template <typename S>
static int norm_t(double* res, const void* a, int64_t len, int m, const Scratch& ws, cudaStream_t st,
                  int fin, BicgScalars* sc) {
    using S2 = typename St<S>::S2;
    const int block = rhs_block(m);
    auto k = norm2_kernel<S>;
    int grid = resident_grid(k, block, len * m);
    if (grid > ws.max_blocks) grid = ws.max_blocks;
    RedArgs ra{ws.partials, ws.counter, ws.result, sc, res, fin};
    k<<<grid, block, 0, st>>>(static_cast<const S2*>(a), len * m, m, ra);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

template <typename S>
static int axpy_t(int op, void* res, const void* sa, const void* x, const void* sb, const void* y,
                  const void* sc, const void* z, int64_t len, int m, cudaStream_t st) {
    using S2 = typename St<S>::S2;
    const int block = rhs_block(m);
    void (*k)(S2*, const double2*, const S2*, const double2*, const S2*, const double2*, const S2*,
              int64_t, int) = nullptr;
    switch (op) {
        case OP_XSAY: k = axpy_kernel<S, OP_XSAY>; break;
        case OP_XPAY: k = axpy_kernel<S, OP_XPAY>; break;
        case OP_AXPBY: k = axpy_kernel<S, OP_AXPBY>; break;
        default: k = axpy_kernel<S, OP_AXPBYPCZ>; break;
    }
    const int grid = resident_grid(k, block, len * m);
    k<<<grid, block, 0, st>>>(static_cast<S2*>(res), static_cast<const double2*>(sa),
                              static_cast<const S2*>(x), static_cast<const double2*>(sb),
                              static_cast<const S2*>(y), static_cast<const double2*>(sc),
                              static_cast<const S2*>(z), len * m, m);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

int mrhs_dotc(double2* res, const void* a, const void* b, int64_t len, int m, int prec,
              const Scratch& ws, cudaStream_t st) {
    return dispatch_prec(prec, [&](auto tag) { return dotc_t<decltype(tag)>(res, a, b, len, m, ws, st); });
}

int mrhs_norm(double* res, const void* a, int64_t len, int m, int prec, const Scratch& ws,
              cudaStream_t st, int fin, BicgScalars* sc) {
    return dispatch_prec(prec, [&](auto tag) { return norm_t<decltype(tag)>(res, a, len, m, ws, st, fin, sc); });
}

int mrhs_axpy(int op, void* res, const void* a, const void* x, const void* b, const void* y,
              const void* c, const void* z, int64_t len, int m, int prec, cudaStream_t st) {
    return dispatch_prec(prec, [&](auto tag) {
        return axpy_t<decltype(tag)>(op, res, a, x, b, y, c, z, len, m, st);
    });
}

// ---------------- m-length scalar kernels ----------------
__global__ void elementwise_kernel(double2* res, const double2* x, const double2* y, int m, int op,
                                   double re, double im) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    if (op == 0) res[j] = cdiv(x[j], y[j]);
    else if (op == 1) res[j] = cmul(x[j], y[j]);
    else res[j] = make_double2(re, im);
}

int elementwise(int op, void* res, const void* x, const void* y, int m, double re, double im,
                cudaStream_t st) {
    if (m < 1) return set_error(QCU_ERR_INVALID, "m=%d", m);
    elementwise_kernel<<<(m + 127) / 128, 128, 0, st>>>(static_cast<double2*>(res),
                                                        static_cast<const double2*>(x),
                                                        static_cast<const double2*>(y), m, op, re, im);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

// ---------------- fused BiCGStab steps ----------------
template <typename S, typename SX>
static int bicg_step_t(int step, const BicgStepArgs& a, cudaStream_t st) {
    using S2 = typename St<S>::S2;
    using X2 = typename St<SX>::S2;
    const int m = a.m;
    const int64_t n = a.len * m;
    const int block = rhs_block(m);
    switch (step) {
        case STEP_INIT: {
            auto k = bicg_init_kernel<S, SX>;
            int grid = resident_grid(k, block, n);
            if (grid > a.ws.max_blocks) grid = a.ws.max_blocks;
            RedArgs ra{a.ws.partials, a.ws.counter, a.ws.result, a.sc, nullptr, FIN_INIT};
            k<<<grid, block, 0, st>>>(static_cast<const S2*>(a.src), static_cast<S2*>(a.r0),
                                      static_cast<S2*>(a.r), static_cast<S2*>(a.p),
                                      static_cast<X2*>(a.x), n, m, ra);
        } break;
        case STEP_S: {
            auto k = bicg_s_kernel<S>;
            const int grid = resident_grid(k, block, n);
            k<<<grid, block, 0, st>>>(static_cast<S2*>(a.s), static_cast<const S2*>(a.r),
                                      static_cast<const S2*>(a.v), a.sc, n, m);
        } break;
        case STEP_XR: {
            auto k = bicg_xr_kernel<S, SX>;
            int grid = resident_grid(k, block, n);
            if (grid > a.ws.max_blocks) grid = a.ws.max_blocks;
            RedArgs ra{a.ws.partials, a.ws.counter, a.ws.result, a.sc, nullptr, FIN_BETA};
            k<<<grid, block, 0, st>>>(static_cast<X2*>(a.x), static_cast<S2*>(a.r),
                                      static_cast<const S2*>(a.p), static_cast<const S2*>(a.s),
                                      static_cast<const S2*>(a.t), static_cast<const S2*>(a.r0), a.sc,
                                      n, m, ra);
        } break;
        case STEP_P: {
            auto k = bicg_p_kernel<S>;
            const int grid = resident_grid(k, block, n);
            k<<<grid, block, 0, st>>>(static_cast<S2*>(a.p), static_cast<const S2*>(a.r),
                                      static_cast<const S2*>(a.v), a.sc, n, m);
        } break;
        default: return set_error(QCU_ERR_INVALID, "unknown bicg step %d", step);
    }
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

int bicg_step(int step, int prec, int x_prec, const BicgStepArgs& a, cudaStream_t st) {
    if (prec == QCU_PRECISION_DOUBLE) {
        if (x_prec != QCU_PRECISION_DOUBLE)
            return set_error(QCU_ERR_INVALID, "FP64 iteration needs an FP64 solution vector");
        return bicg_step_t<double, double>(step, a, st);
    }
    if (x_prec != QCU_PRECISION_SINGLE)
        return set_error(QCU_ERR_INVALID, "sloppy iteration accumulates the solution in FP32");
    switch (prec) {
        case QCU_PRECISION_SINGLE: return bicg_step_t<float, float>(step, a, st);
        case QCU_PRECISION_HALF: return bicg_step_t<__half, float>(step, a, st);
        case QCU_PRECISION_BF16: return bicg_step_t<__nv_bfloat16, float>(step, a, st);
        default: return set_error(QCU_ERR_INVALID, "precision %d", prec);
    }
}

// ---------------- mixed precision reliable updates ----------------
int mp_accum(void* x64, void* e, BicgScalars* sc, int64_t len, int m, cudaStream_t st) {
    const int block = rhs_block(m);
    const int grid = resident_grid(mp_accum_kernel, block, len * m);
    mp_accum_kernel<<<grid, block, 0, st>>>(static_cast<double2*>(x64), static_cast<const float2*>(e), sc,
                                            len * m, m);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

template <typename S>
static int mp_load_t(void* rs, void* ps, void* r0s, const void* r64, BicgScalars* sc, int64_t len,
                     int m, int init, const Scratch& ws, cudaStream_t st) {
    using S2 = typename St<S>::S2;
    const int block = rhs_block(m);
    auto k = mp_load_kernel<S>;
    int grid = resident_grid(k, block, len * m);
    if (grid > ws.max_blocks) grid = ws.max_blocks;
    RedArgs ra{ws.partials, ws.counter, ws.result, sc, nullptr, FIN_RHO};
    k<<<grid, block, 0, st>>>(static_cast<S2*>(rs), static_cast<S2*>(ps), static_cast<S2*>(r0s),
                              static_cast<const double2*>(r64), sc, len * m, m, init, ra);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

int mp_load(int prec, void* rs, void* ps, void* r0s, const void* r64, BicgScalars* sc, int64_t len,
            int m, int init, const Scratch& ws, cudaStream_t st) {
    return dispatch_prec(prec, [&](auto tag) {
        return mp_load_t<decltype(tag)>(rs, ps, r0s, r64, sc, len, m, init, ws, st);
    });
}

int mp_update(BicgScalars* sc, int m, int init, cudaStream_t st) {
    mp_update_kernel<<<1, 64, 0, st>>>(sc, m, init);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

}  // namespace qcub
