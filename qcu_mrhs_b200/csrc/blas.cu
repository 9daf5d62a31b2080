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
// ---- two RHS per thread for 16-bit storage (m even) ----
// Thread per RHS pair: RHS 2q and 2q+1 of an element are adjacent, so every 16-bit vector
// is read and written as 8-byte words and the FP32 increment as 16-byte words (the per-RHS
// kernels move 4 and 8 bytes per access).  Same per-element arithmetic as bicg_*_kernel;
// per-thread FP32 partial sums, FP64 across threads and blocks in a fixed order.
namespace {

template <typename S>
__device__ __forceinline__ float2 ld16(uint32_t w) {
    return St<S>::ld(*reinterpret_cast<const typename St<S>::S2*>(&w));
}
template <typename S>
__device__ __forceinline__ uint32_t st16(float2 v) {
    const typename St<S>::S2 h = St<S>::cv(v);
    return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Block + grid reduction when thread t holds the sums of RHS 2 (t % (m/2)) and 2 (t % (m/2)) + 1.
template <int NV>
__device__ inline void grid_reduce_rhs_pairs(const double2 (&v)[2][NV], int m, const RedArgs& ra) {
    __shared__ double2 sh[NV][2][kRedThreads];
    __shared__ double2 bsum[NV * kMaxRhs];
    const int tid = threadIdx.x, nb = blockDim.x, half = m >> 1;
#pragma unroll
    for (int k = 0; k < NV; ++k)
#pragma unroll
        for (int q = 0; q < 2; ++q) sh[k][q][tid] = v[q][k];
    __syncthreads();
    for (int idx = tid; idx < NV * m; idx += nb) {
        const int k = idx / m, rhs = idx - k * m;
        const int jp = rhs >> 1, q = rhs & 1;
        double2 acc = make_double2(0.0, 0.0);
        for (int t = jp; t < nb; t += half) {
            acc.x += sh[k][q][t].x;
            acc.y += sh[k][q][t].y;
        }
        bsum[idx] = acc;
    }
    __syncthreads();
    publish_and_finish<NV>(bsum, m, ra);
}

#define QCUB_PAIR_LOOP(gi, np)                                                               \
    for (int64_t gi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gi < (np);           \
         gi += (int64_t)gridDim.x * blockDim.x)

// s = r - alpha v
template <typename S>
__global__ void __launch_bounds__(kRedThreads)
bicg_s2_kernel(uint2* __restrict__ s, const uint2* __restrict__ r, const uint2* __restrict__ v,
               const BicgScalars* __restrict__ sc, int64_t np, int m) {
    if (sc->done) return;
    const int jp = threadIdx.x % (m >> 1);
    const float2 al0 = from_d2<float2>(sc->alpha[2 * jp]), al1 = from_d2<float2>(sc->alpha[2 * jp + 1]);
    QCUB_PAIR_LOOP(gi, np) {
        const uint2 rw = r[gi], vw = v[gi];
        const float2 r0 = ld16<S>(rw.x), r1 = ld16<S>(rw.y);
        const float2 a0 = cmulf(al0, ld16<S>(vw.x)), a1 = cmulf(al1, ld16<S>(vw.y));
        s[gi] = make_uint2(st16<S>(make_float2(r0.x - a0.x, r0.y - a0.y)),
                           st16<S>(make_float2(r1.x - a1.x, r1.y - a1.y)));
    }
}

// x += alpha p + omega s ; r = s - omega t ; reduce |r|^2, <r0, r>  (FIN_BETA);
// with sc->x_fresh, x = alpha p + omega s
template <typename S>
__global__ void __launch_bounds__(kRedThreads)
bicg_xr2_kernel(float4* __restrict__ x, uint2* __restrict__ r, const uint2* __restrict__ p,
                const uint2* __restrict__ s, const uint2* __restrict__ t, const uint2* __restrict__ r0,
                const BicgScalars* __restrict__ sc, int64_t np, int m, RedArgs ra) {
    if (sc->done) return;
    const int jp = threadIdx.x % (m >> 1);
    float2 al[2], om[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        al[q] = from_d2<float2>(sc->alpha[2 * jp + q]);
        om[q] = from_d2<float2>(sc->omega[2 * jp + q]);
    }
    float v[2][2][2] = {{{0.f, 0.f}, {0.f, 0.f}}, {{0.f, 0.f}, {0.f, 0.f}}};   // [rhs][sum][re, im]
    const bool fresh = sc->x_fresh != 0;
    QCUB_PAIR_LOOP(gi, np) {
        const uint2 pw = p[gi], sw = s[gi], tw = t[gi], qw = r0[gi];
        const float4 xo = fresh ? make_float4(0.f, 0.f, 0.f, 0.f) : x[gi];
        float xs[4] = {xo.x, xo.y, xo.z, xo.w};
        uint32_t rb[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const float2 pv = ld16<S>(q ? pw.y : pw.x), sv = ld16<S>(q ? sw.y : sw.x);
            const float2 tv = ld16<S>(q ? tw.y : tw.x);
            const float2 ap = cmulf(al[q], pv), os = cmulf(om[q], sv);
            xs[2 * q] += ap.x + os.x;
            xs[2 * q + 1] += ap.y + os.y;
            const float2 ot = cmulf(om[q], tv);
            rb[q] = st16<S>(make_float2(sv.x - ot.x, sv.y - ot.y));
            const float2 rv = ld16<S>(rb[q]);
            const float2 qv = ld16<S>(q ? qw.y : qw.x);
            v[q][0][0] += rv.x * rv.x + rv.y * rv.y;
            v[q][1][0] += qv.x * rv.x + qv.y * rv.y;
            v[q][1][1] += qv.x * rv.y - qv.y * rv.x;
        }
        x[gi] = make_float4(xs[0], xs[1], xs[2], xs[3]);
        r[gi] = make_uint2(rb[0], rb[1]);
    }
    double2 d[2][2];
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int k = 0; k < 2; ++k) d[q][k] = make_double2((double)v[q][k][0], (double)v[q][k][1]);
    grid_reduce_rhs_pairs<2>(d, m, ra);
}

// p = r + beta (p - omega v); clears x_fresh (the STEP_XR before it has read it)
template <typename S>
__global__ void __launch_bounds__(kRedThreads)
bicg_p2_kernel(uint2* __restrict__ p, const uint2* __restrict__ r, const uint2* __restrict__ v,
               BicgScalars* __restrict__ sc, int64_t np, int m) {
    if (sc->done) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->x_fresh = 0;
    const int jp = threadIdx.x % (m >> 1);
    float2 be[2], om[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        be[q] = from_d2<float2>(sc->beta[2 * jp + q]);
        om[q] = from_d2<float2>(sc->omega[2 * jp + q]);
    }
    QCUB_PAIR_LOOP(gi, np) {
        const uint2 pw = p[gi], vw = v[gi], rw = r[gi];
        uint32_t ob[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const float2 pv = ld16<S>(q ? pw.y : pw.x);
            const float2 ov = cmulf(om[q], ld16<S>(q ? vw.y : vw.x));
            const float2 bd = cmulf(be[q], make_float2(pv.x - ov.x, pv.y - ov.y));
            const float2 rv = ld16<S>(q ? rw.y : rw.x);
            ob[q] = st16<S>(make_float2(rv.x + bd.x, rv.y + bd.y));
        }
        p[gi] = make_uint2(ob[0], ob[1]);
    }
}

// mp_load_kernel on RHS pairs: the FP64 residual as two 16-byte words, the sloppy vectors
// as 8-byte words; same arithmetic and reduction (FIN_RHO)
template <typename S>
__global__ void __launch_bounds__(kRedThreads)
mp_load2_kernel(uint2* __restrict__ rs, uint2* __restrict__ ps, uint2* __restrict__ r0s,
                const double2* __restrict__ r64, const BicgScalars* __restrict__ sc, int64_t np, int m, int init,
                RedArgs ra) {
    if (!init && mp_skip(sc)) return;
    const bool reset = init || sc->restart;
    const int jp = threadIdx.x % (m >> 1);
    double sj[2];
    float rat[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        sj[q] = sc->scale[2 * jp + q];
        rat[q] = (float)sc->ratio[2 * jp + q];
    }
    double2 v[2][1] = {{make_double2(0.0, 0.0)}, {make_double2(0.0, 0.0)}};
    QCUB_PAIR_LOOP(gi, np) {
        const double2 ra0 = r64[2 * gi], ra1 = r64[2 * gi + 1];
        const uint2 pw = reset ? make_uint2(0u, 0u) : ps[gi];
        const uint2 qw = reset ? make_uint2(0u, 0u) : r0s[gi];
        uint32_t rb[2], pb[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const double2 rv = q ? ra1 : ra0;
            rb[q] = st16<S>(make_float2((float)(sj[q] * rv.x), (float)(sj[q] * rv.y)));
            float2 qv;
            if (reset) {
                pb[q] = rb[q];
                qv = ld16<S>(rb[q]);
            } else {
                const float2 pv = ld16<S>(q ? pw.y : pw.x);
                pb[q] = st16<S>(make_float2(pv.x * rat[q], pv.y * rat[q]));
                qv = ld16<S>(q ? qw.y : qw.x);
            }
            const float2 rr = ld16<S>(rb[q]);
            v[q][0].x += (double)qv.x * rr.x + (double)qv.y * rr.y;
            v[q][0].y += (double)qv.x * rr.y - (double)qv.y * rr.x;
        }
        rs[gi] = make_uint2(rb[0], rb[1]);
        ps[gi] = make_uint2(pb[0], pb[1]);
        if (reset) r0s[gi] = make_uint2(rb[0], rb[1]);
    }
    grid_reduce_rhs_pairs<1>(v, m, ra);
}

bool aligned(const void* ptr, uintptr_t a) { return (reinterpret_cast<uintptr_t>(ptr) % a) == 0; }

// S, XR and P steps for 16-bit storage on RHS pairs; returns -1 where they do not apply
template <typename S>
int bicg_step_pairs(int step, const BicgStepArgs& a, cudaStream_t st) {
    const int m = a.m;
    if (m % 2 || m < 2) return -1;
    const int64_t np = a.len * m / 2;
    const int block = rhs_block(m / 2);
    switch (step) {
        case STEP_S: {
            if (!aligned(a.s, 8) || !aligned(a.r, 8) || !aligned(a.v, 8)) return -1;
            auto k = bicg_s2_kernel<S>;
            const int grid = resident_grid(k, block, np);
            k<<<grid, block, 0, st>>>(static_cast<uint2*>(a.s), static_cast<const uint2*>(a.r),
                                      static_cast<const uint2*>(a.v), a.sc, np, m);
        } break;
        case STEP_XR: {
            if (!aligned(a.x, 16) || !aligned(a.r, 8) || !aligned(a.p, 8) || !aligned(a.s, 8) ||
                !aligned(a.t, 8) || !aligned(a.r0, 8))
                return -1;
            auto k = bicg_xr2_kernel<S>;
            int grid = resident_grid(k, block, np);
            if (grid > a.ws.max_blocks) grid = a.ws.max_blocks;
            RedArgs ra{a.ws.partials, a.ws.counter, a.ws.result, a.sc, nullptr, FIN_BETA};
            k<<<grid, block, 0, st>>>(static_cast<float4*>(a.x), static_cast<uint2*>(a.r),
                                      static_cast<const uint2*>(a.p), static_cast<const uint2*>(a.s),
                                      static_cast<const uint2*>(a.t), static_cast<const uint2*>(a.r0), a.sc,
                                      np, m, ra);
        } break;
        case STEP_P: {
            if (!aligned(a.p, 8) || !aligned(a.r, 8) || !aligned(a.v, 8)) return -1;
            auto k = bicg_p2_kernel<S>;
            const int grid = resident_grid(k, block, np);
            k<<<grid, block, 0, st>>>(static_cast<uint2*>(a.p), static_cast<const uint2*>(a.r),
                                      static_cast<const uint2*>(a.v), a.sc, np, m);
        } break;
        default: return -1;
    }
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

}  // namespace

template <typename S, typename SX>
static int bicg_step_t(int step, const BicgStepArgs& a, cudaStream_t st) {
    using S2 = typename St<S>::S2;
    using X2 = typename St<SX>::S2;
    const int m = a.m;
    const int64_t n = a.len * m;
    const int block = rhs_block(m);
    if constexpr (sizeof(S) == 2) {
        const int rc = bicg_step_pairs<S>(step, a, st);
        if (rc >= 0) return rc;
    }
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
    if constexpr (sizeof(S) == 2) {
        if (m % 2 == 0 && aligned(rs, 8) && aligned(ps, 8) && aligned(r0s, 8) && aligned(r64, 16)) {
            const int block = rhs_block(m / 2);
            const int64_t np = len * m / 2;
            auto k = mp_load2_kernel<S>;
            int grid = resident_grid(k, block, np);
            if (grid > ws.max_blocks) grid = ws.max_blocks;
            RedArgs ra{ws.partials, ws.counter, ws.result, sc, nullptr, FIN_RHO};
            k<<<grid, block, 0, st>>>(static_cast<uint2*>(rs), static_cast<uint2*>(ps), static_cast<uint2*>(r0s),
                                      static_cast<const double2*>(r64), sc, np, m, init, ra);
            QCUB_CHECK_LAUNCH();
            return QCU_SUCCESS;
        }
    }
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
