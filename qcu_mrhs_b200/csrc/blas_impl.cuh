// blas_impl.cuh -- multi-RHS BLAS kernels on strided vectors (element i of RHS j at
// complex offset i*m + j) and the fused BiCGStab update steps built from them.
//
// Reference operators (one launch per RHS there, one launch for all RHS here):
//   dotc      src/qcu_blas/qcu_complex_dotc.cu:20-75     res_j = sum_i conj(a_ij) b_ij
//   norm      src/qcu_blas/qcu_complex_norm.cu:20-57      res_j = sqrt(sum_i |a_ij|^2)
//   xsay      include/kernel/element_wise/c_xsay.cuh      res = x - a_j y
//   xpay      include/kernel/element_wise/c_xpay.cuh      res = x + a_j y
//   axpby     include/kernel/element_wise/c_axpby.cuh     res = a_j x + b_j y
//   axpbypcz  include/kernel/element_wise/c_axpbypcz.cuh  res = a_j x + b_j y + c_j z
// The block size is a multiple of m and the grid stride is a multiple of m, so each
// thread keeps one RHS and reads its scalars once.
#pragma once

#include "blas.h"
#include "dslash_impl.cuh"
#include "reduce.cuh"

namespace qcub {

template <typename A2>
__device__ __forceinline__ A2 cmulA(const A2& a, const A2& b) {
    return mk2<A2>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename A2>
__device__ __forceinline__ A2 from_d2(double2 v) {
    return mk2<A2>((decltype(A2::x))v.x, (decltype(A2::x))v.y);
}

// Per-thread partial sums of the solver's fused reductions: FP32 for 16-bit storage (the
// inputs carry 1e-3 relative noise), FP64 otherwise; the sums across threads and blocks
// are FP64.  The standalone dotc / norm kernels keep FP64 partials at every precision.
template <typename S> struct RedAcc { using T = double; };
template <> struct RedAcc<__half> { using T = float; };
template <> struct RedAcc<__nv_bfloat16> { using T = float; };

template <typename R, int NV>
__device__ __forceinline__ void reduce_partials(const R (&v)[NV][2], int m, const RedArgs& ra) {
    double2 d[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) d[k] = make_double2((double)v[k][0], (double)v[k][1]);
    grid_reduce<NV>(d, m, ra);
}

#define QCUB_GRID_LOOP(gi, n)                                                                \
    for (int64_t gi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gi < (n);            \
         gi += (int64_t)gridDim.x * blockDim.x)

template <typename S>
__global__ void __launch_bounds__(kRedThreads) dotc_kernel(const typename St<S>::S2* __restrict__ a,
                                                           const typename St<S>::S2* __restrict__ b,
                                                           int64_t n, int m, RedArgs ra) {
    using R = double;   // the standalone reductions keep FP64 partial sums at every precision
    R v[1][2] = {{0, 0}};
    QCUB_GRID_LOOP(gi, n) {
        const auto x = St<S>::ld(a[gi]);
        const auto y = St<S>::ld(b[gi]);
        v[0][0] += (R)x.x * y.x + (R)x.y * y.y;
        v[0][1] += (R)x.x * y.y - (R)x.y * y.x;
    }
    reduce_partials<R, 1>(v, m, ra);
}

template <typename S>
__global__ void __launch_bounds__(kRedThreads) norm2_kernel(const typename St<S>::S2* __restrict__ a,
                                                            int64_t n, int m, RedArgs ra) {
    using R = double;   // the standalone reductions keep FP64 partial sums at every precision
    R v[1][2] = {{0, 0}};
    QCUB_GRID_LOOP(gi, n) {
        const auto x = St<S>::ld(a[gi]);
        v[0][0] += (R)x.x * x.x + (R)x.y * x.y;
    }
    reduce_partials<R, 1>(v, m, ra);
}

template <typename S, int OP>
__global__ void __launch_bounds__(kRedThreads)
axpy_kernel(typename St<S>::S2* __restrict__ res, const double2* __restrict__ sa,
            const typename St<S>::S2* __restrict__ x, const double2* __restrict__ sb,
            const typename St<S>::S2* __restrict__ y, const double2* __restrict__ sc,
            const typename St<S>::S2* __restrict__ z, int64_t n, int m) {
    using A2 = typename St<S>::A2;
    const int j = threadIdx.x % m;
    const A2 a = from_d2<A2>(sa[j]);
    const A2 b = (OP >= OP_AXPBY) ? from_d2<A2>(sb[j]) : mk2<A2>(0, 0);
    const A2 c = (OP == OP_AXPBYPCZ) ? from_d2<A2>(sc[j]) : mk2<A2>(0, 0);
    QCUB_GRID_LOOP(gi, n) {
        const A2 xv = St<S>::ld(x[gi]);
        const A2 yv = St<S>::ld(y[gi]);
        A2 r;
        if (OP == OP_XSAY) {
            const A2 ay = cmulA(a, yv);
            r = mk2<A2>(xv.x - ay.x, xv.y - ay.y);
        } else if (OP == OP_XPAY) {
            const A2 ay = cmulA(a, yv);
            r = mk2<A2>(xv.x + ay.x, xv.y + ay.y);
        } else {
            const A2 ax = cmulA(a, xv), by = cmulA(b, yv);
            r = mk2<A2>(ax.x + by.x, ax.y + by.y);
            if (OP == OP_AXPBYPCZ) {
                const A2 cz = cmulA(c, St<S>::ld(z[gi]));
                r.x += cz.x;
                r.y += cz.y;
            }
        }
        res[gi] = St<S>::cv(r);
    }
}

// ---------------- fused BiCGStab steps (reference bicgstab_solve.cu:252-386) ----------------

// r0 = r = p = src ; x = 0 ; reduce |src|^2 (FIN_INIT: rho = ||b'||^2, bnorm2)
template <typename S, typename SX>
__global__ void __launch_bounds__(kRedThreads)
bicg_init_kernel(const typename St<S>::S2* __restrict__ src, typename St<S>::S2* __restrict__ r0,
                 typename St<S>::S2* __restrict__ r, typename St<S>::S2* __restrict__ p,
                 typename St<SX>::S2* __restrict__ x, int64_t n, int m, RedArgs ra) {
    double2 v[1] = {make_double2(0.0, 0.0)};
    QCUB_GRID_LOOP(gi, n) {
        const auto sv = src[gi];
        r0[gi] = sv;
        r[gi] = sv;
        p[gi] = sv;
        if (x != nullptr) x[gi] = St<SX>::cv(mk2<typename St<SX>::A2>(0, 0));
        const auto a = St<S>::ld(sv);
        v[0].x += (double)a.x * a.x + (double)a.y * a.y;
    }
    grid_reduce<1>(v, m, ra);
}

// s = r - alpha v
template <typename S>
__global__ void __launch_bounds__(kRedThreads)
bicg_s_kernel(typename St<S>::S2* __restrict__ s, const typename St<S>::S2* __restrict__ r,
              const typename St<S>::S2* __restrict__ v, const BicgScalars* __restrict__ sc, int64_t n,
              int m) {
    using A2 = typename St<S>::A2;
    if (sc->done) return;
    const int j = threadIdx.x % m;
    const A2 al = from_d2<A2>(sc->alpha[j]);
    QCUB_GRID_LOOP(gi, n) {
        const A2 rv = St<S>::ld(r[gi]);
        const A2 av = cmulA(al, St<S>::ld(v[gi]));
        s[gi] = St<S>::cv(mk2<A2>(rv.x - av.x, rv.y - av.y));
    }
}

// x += alpha p + omega s ; r = s - omega t ; reduce |r|^2, <r0, r>  (FIN_BETA).
// With sc->x_fresh (mixed solver, first step after a reliable update) x = alpha p + omega s.
template <typename S, typename SX>
__global__ void __launch_bounds__(kRedThreads)
bicg_xr_kernel(typename St<SX>::S2* __restrict__ x, typename St<S>::S2* __restrict__ r,
               const typename St<S>::S2* __restrict__ p, const typename St<S>::S2* __restrict__ s,
               const typename St<S>::S2* __restrict__ t, const typename St<S>::S2* __restrict__ r0,
               const BicgScalars* __restrict__ sc, int64_t n, int m, RedArgs ra) {
    using A2 = typename St<S>::A2;
    using X2 = typename St<SX>::A2;
    if (sc->done) return;
    const int j = threadIdx.x % m;
    const X2 al = from_d2<X2>(sc->alpha[j]);
    const X2 om = from_d2<X2>(sc->omega[j]);
    const A2 omA = from_d2<A2>(sc->omega[j]);
    using R = typename RedAcc<S>::T;
    R v[2][2] = {{0, 0}, {0, 0}};
    const bool fresh = sc->x_fresh != 0;
    QCUB_GRID_LOOP(gi, n) {
        const A2 pv = St<S>::ld(p[gi]);
        const A2 sv = St<S>::ld(s[gi]);
        const A2 tv = St<S>::ld(t[gi]);
        X2 xv = fresh ? mk2<X2>(0, 0) : St<SX>::ld(x[gi]);
        const X2 ap = cmulA(al, mk2<X2>(pv.x, pv.y));
        const X2 os = cmulA(om, mk2<X2>(sv.x, sv.y));
        xv.x += ap.x + os.x;
        xv.y += ap.y + os.y;
        x[gi] = St<SX>::cv(xv);
        const A2 ot = cmulA(omA, tv);
        const typename St<S>::S2 rs = St<S>::cv(mk2<A2>(sv.x - ot.x, sv.y - ot.y));
        r[gi] = rs;
        const A2 rv = St<S>::ld(rs);
        const A2 q = St<S>::ld(r0[gi]);
        v[0][0] += (R)rv.x * rv.x + (R)rv.y * rv.y;
        v[1][0] += (R)q.x * rv.x + (R)q.y * rv.y;
        v[1][1] += (R)q.x * rv.y - (R)q.y * rv.x;
    }
    reduce_partials<R, 2>(v, m, ra);
}

// p = r + beta (p - omega v); clears x_fresh (the STEP_XR before it has read it)
template <typename S>
__global__ void __launch_bounds__(kRedThreads)
bicg_p_kernel(typename St<S>::S2* __restrict__ p, const typename St<S>::S2* __restrict__ r,
              const typename St<S>::S2* __restrict__ v, BicgScalars* __restrict__ sc, int64_t n,
              int m) {
    using A2 = typename St<S>::A2;
    if (sc->done) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->x_fresh = 0;
    const int j = threadIdx.x % m;
    const A2 be = from_d2<A2>(sc->beta[j]);
    const A2 om = from_d2<A2>(sc->omega[j]);
    QCUB_GRID_LOOP(gi, n) {
        const A2 pv = St<S>::ld(p[gi]);
        const A2 ov = cmulA(om, St<S>::ld(v[gi]));
        const A2 d = mk2<A2>(pv.x - ov.x, pv.y - ov.y);
        const A2 bd = cmulA(be, d);
        const A2 rv = St<S>::ld(r[gi]);
        p[gi] = St<S>::cv(mk2<A2>(rv.x + bd.x, rv.y + bd.y));
    }
}

// ---------------- mixed precision: FP64 reliable updates ----------------

__device__ __forceinline__ bool mp_skip(const BicgScalars* sc) { return sc->done || !sc->gate; }

// x64 += e / scale_j (gated by a pending reliable update); e is not zeroed: x_fresh makes
// the next STEP_XR overwrite it.  Non-finite elements of e (a sloppy iterate that overflowed
// before the breakdown was caught) are dropped, so x64 stays finite and the restart
// continues from it.
static __global__ void __launch_bounds__(kRedThreads)
mp_accum_kernel(double2* __restrict__ x64, const float2* __restrict__ e, BicgScalars* __restrict__ sc,
                int64_t n, int m) {
    if (mp_skip(sc)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->x_fresh = 1;
    const int j = threadIdx.x % m;
    const double inv = 1.0 / sc->scale[j];
    QCUB_GRID_LOOP(gi, n) {
        const float2 ev = e[gi];
        if (isfinite(ev.x) && isfinite(ev.y)) {
            double2 xv = x64[gi];
            xv.x += inv * ev.x;
            xv.y += inv * ev.y;
            x64[gi] = xv;
        }
    }
}

// New sloppy residual from the FP64 residual: rs = scale_j * r64.  With init (or a
// pending restart): r0s = ps = rs; otherwise ps *= ratio_j.  Reduces <r0s, rs> -> rho.
template <typename S>
__global__ void __launch_bounds__(kRedThreads)
mp_load_kernel(typename St<S>::S2* __restrict__ rs, typename St<S>::S2* __restrict__ ps,
               typename St<S>::S2* __restrict__ r0s, const double2* __restrict__ r64,
               const BicgScalars* __restrict__ sc, int64_t n, int m, int init, RedArgs ra) {
    using A2 = typename St<S>::A2;
    using A = typename St<S>::A;
    if (!init && mp_skip(sc)) return;
    const bool reset = init || sc->restart;
    const int j = threadIdx.x % m;
    const double sj = sc->scale[j];
    const A rat = (A)sc->ratio[j];
    double2 v[1] = {make_double2(0.0, 0.0)};
    QCUB_GRID_LOOP(gi, n) {
        const double2 rv = r64[gi];
        const typename St<S>::S2 rst = St<S>::cv(mk2<A2>((A)(sj * rv.x), (A)(sj * rv.y)));
        rs[gi] = rst;
        A2 q;
        if (reset) {
            ps[gi] = rst;
            r0s[gi] = rst;
            q = St<S>::ld(rst);
        } else {
            const A2 pv = St<S>::ld(ps[gi]);
            ps[gi] = St<S>::cv(mk2<A2>(pv.x * rat, pv.y * rat));
            q = St<S>::ld(r0s[gi]);
        }
        const A2 rr = St<S>::ld(rst);
        v[0].x += (double)q.x * rr.x + (double)q.y * rr.y;
        v[0].y += (double)q.x * rr.y - (double)q.y * rr.x;
    }
    grid_reduce<1>(v, m, ra);
}

// One block: decide convergence from the FP64 true residual and rescale.
// init: first call (sets scale from ||r64|| without touching counters).
static __global__ void mp_update_kernel(BicgScalars* sc, int m, int init) {
    if (!init && mp_skip(sc)) return;
    __shared__ int all_conv, stalled;
    if (threadIdx.x == 0) { all_conv = 1; stalled = 0; }
    __syncthreads();
    const int j = threadIdx.x;
    if (j < m) {
        const double r2 = sc->rtrue2[j];
        const bool conv = r2 <= sc->tol2 * sc->bfull2[j];
        if (init) {
            sc->best2[j] = r2;
            sc->stall[j] = 0;
        } else if (sc->active[j] && !conv) {
            if (r2 < 0.98 * sc->best2[j]) {
                sc->best2[j] = r2;
                sc->stall[j] = 0;
            } else if (++sc->stall[j] >= kStallUpdates) {
                atomicOr(&stalled, 1);
            }
        }
        if (conv) sc->active[j] = 0;
        if (!conv) atomicAnd(&all_conv, 0);
        // scale so that the sloppy residual has unit RMS element (O(1) values keep FP16
        // away from its subnormal range as the residual shrinks)
        const double rn = sqrt(r2);
        const double nrm = sqrt(sc->len_per_rhs);
        const double snew = (rn > 0.0 && isfinite(rn)) ? nrm / rn : 1.0;
        sc->ratio[j] = snew / sc->scale[j];
        sc->scale[j] = snew;
        sc->maxr[j] = nrm;
        sc->rnorm2[j] = nrm * nrm;
        if (!isfinite(r2)) atomicAnd(&all_conv, 0);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (!init) sc->reliable += 1;
        if (all_conv) {
            sc->status = 1;
            sc->done = 1;
        } else if (stalled) {
            sc->status = 4;
            sc->done = 1;
        }
    }
}

}  // namespace qcub
