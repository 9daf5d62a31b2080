// precond.cu -- kernels and host code of the learned gauge-covariant preconditioner
// (precond.h): the parallel-transport convolution layer, its adjoint (the same kernel
// with conjugate-transposed spin weights and reversed hops, since T_{+mu}^dag = T_{-mu}),
// the weight gradient, Adam, the training loss ||M P b - b||^2 / ||b||^2, and the FP64
// kernels of the right-preconditioned BiCGStab.
//
// No reference code: the preconditioner is new in this library.  Its CPU restatement
// (oracle_ptc_forward / _adjoint / _wgrad) is the checker of these kernels.
#include <cmath>
#include <cstring>

#include "blas.h"
#include "dslash.h"
#include "layout.h"
#include "precond.h"

namespace qcub {

int sm_count();

namespace {

constexpr int kPaths = 9;
constexpr int kPtcThreads = 256;

__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 c) {   // c + a b
    c.x = fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x));
    c.y = fmaf(a.x, b.y, fmaf(a.y, b.x, c.y));
    return c;
}

// Path k of full-lattice site `site` (= parity * vh + half index): source site and link
// (index into the [4][2][Vh] link array; forward links are used as is, backward links
// conjugate-transposed), and the t-boundary factor.
__device__ __forceinline__ void ptc_path(const Geom& g, int64_t site, int k, float t_sign, int64_t* src,
                                         int64_t* link, bool* fwd, float* sg) {
    const int64_t vh = g.vh;
    const int p = site >= vh ? 1 : 0;
    const int64_t idx = site - p * vh;
    *sg = 1.f;
    *fwd = true;
    *link = 0;
    if (k == 0) {
        *src = site;
        return;
    }
    const int mu = (k - 1) >> 1;
    const bool f = ((k - 1) & 1) == 0;
    const SiteXYZT c = site_coords(g, (uint32_t)idx);
    const int lxh = g.lxh, Ly = g.L[1], Lz = g.L[2], Lt = g.L[3];
    const int64_t sy = lxh, sz = (int64_t)lxh * Ly, st = sz * Lz;
    int64_t nb;
    bool wrap = false;
    if (mu == 0) {
        const int xodd = (p ^ (c.y + c.z + c.t)) & 1;
        nb = f ? idx - c.xh + (xodd ? (c.xh + 1 == lxh ? 0 : c.xh + 1) : c.xh)
               : idx - c.xh + (xodd ? c.xh : (c.xh == 0 ? lxh - 1 : c.xh - 1));
    } else if (mu == 1) {
        nb = f ? idx + (c.y + 1 == Ly ? -(int64_t)(Ly - 1) * sy : sy) : idx + (c.y == 0 ? (int64_t)(Ly - 1) * sy : -sy);
    } else if (mu == 2) {
        nb = f ? idx + (c.z + 1 == Lz ? -(int64_t)(Lz - 1) * sz : sz) : idx + (c.z == 0 ? (int64_t)(Lz - 1) * sz : -sz);
    } else {
        wrap = f ? (c.t + 1 == Lt) : (c.t == 0);
        nb = f ? idx + (wrap ? -(int64_t)(Lt - 1) * st : st) : idx + (wrap ? (int64_t)(Lt - 1) * st : -st);
    }
    *src = (int64_t)(1 - p) * vh + nb;
    *link = f ? ((int64_t)(mu * 2 + p) * vh + idx) : ((int64_t)(mu * 2 + (1 - p)) * vh + nb);
    *fwd = f;
    *sg = wrap ? t_sign : 1.f;
}

// tv = (T_k f)(site) for RHS r: f points at the channel's field + r
template <int NC>
__device__ __forceinline__ void ptc_transport(float2 (&tv)[4][NC], const float2* __restrict__ f,
                                              const float2* __restrict__ gauge, const Geom& g, int64_t site,
                                              int k, float t_sign, int m) {
    const int64_t slen = 4 * NC * (int64_t)m;
    int64_t src, link;
    bool fwd;
    float sg;
    ptc_path(g, site, k, t_sign, &src, &link, &fwd, &sg);
    const float2* v = f + src * slen;
    if (k == 0) {
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
            for (int c = 0; c < NC; ++c) tv[s][c] = v[(s * NC + c) * m];
        return;
    }
    const float2* U = gauge + link * (NC * NC);
    float2 u[NC][NC];
#pragma unroll
    for (int a = 0; a < NC; ++a)
#pragma unroll
        for (int b = 0; b < NC; ++b) {
            const float2 e = fwd ? U[a * NC + b] : U[b * NC + a];
            u[a][b] = make_float2(sg * e.x, fwd ? sg * e.y : -sg * e.y);
        }
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        float2 in[NC];
#pragma unroll
        for (int b = 0; b < NC; ++b) in[b] = v[(s * NC + b) * m];
#pragma unroll
        for (int a = 0; a < NC; ++a) {
            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
            for (int b = 0; b < NC; ++b) acc = cfma(u[a][b], in[b], acc);
            tv[s][a] = acc;
        }
    }
}

// One layer: out_o = sum_i sum_k W[o][i][k] T_k in_i.  Thread per (site, o, r); the
// layer's weights are staged in shared memory.
template <int NC>
__global__ void __launch_bounds__(kPtcThreads)
ptc_layer_kernel(float2* __restrict__ out, const float2* __restrict__ in, const float2* __restrict__ w,
                 const float2* __restrict__ gauge, Geom g, int m, int cin, int cout, float t_sign,
                 const int* __restrict__ done) {
    if (done != nullptr && *done) return;
    extern __shared__ float2 sw[];
    const int nw = cout * cin * kPaths * 16;
    for (int e = threadIdx.x; e < nw; e += blockDim.x) sw[e] = w[e];
    __syncthreads();
    const int per = m * cout;
    const int spb = blockDim.x / per;
    if ((int)threadIdx.x >= spb * per) return;
    const int r = threadIdx.x % m;
    const int o = (threadIdx.x / m) % cout;
    const int64_t slen = 4 * NC * (int64_t)m;
    const int64_t field = 2 * g.vh * slen;
    for (int64_t site = (int64_t)blockIdx.x * spb + threadIdx.x / per; site < 2 * g.vh;
         site += (int64_t)gridDim.x * spb) {
        float2 acc[4][NC];
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
            for (int c = 0; c < NC; ++c) acc[s][c] = make_float2(0.f, 0.f);
        for (int k = 0; k < kPaths; ++k) {
            for (int i = 0; i < cin; ++i) {
                float2 tv[4][NC];
                ptc_transport<NC>(tv, in + i * field + r, gauge, g, site, k, t_sign, m);
                const float2* W = sw + ((o * cin + i) * kPaths + k) * 16;
#pragma unroll
                for (int sp = 0; sp < 4; ++sp)
#pragma unroll
                    for (int s = 0; s < 4; ++s) {
                        const float2 wv = W[sp * 4 + s];
#pragma unroll
                        for (int c = 0; c < NC; ++c) acc[sp][c] = cfma(wv, tv[s][c], acc[sp][c]);
                    }
            }
        }
        float2* dst = out + o * field + site * slen + r;
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
            for (int c = 0; c < NC; ++c) dst[(s * NC + c) * m] = acc[s][c];
    }
}

// gw[o][i][k][s'][s] = sum_{site, c, r} gout_o[s'][c][r] conj((T_k in_i)[s][c][r]); one block
// per (o, i, k), fixed thread-to-element assignment and a fixed reduction order.
template <int NC>
__global__ void __launch_bounds__(kPtcThreads)
ptc_wgrad_kernel(double2* __restrict__ gw, const float2* __restrict__ gout, const float2* __restrict__ in,
                 const float2* __restrict__ gauge, Geom g, int m, int cin, int cout, float t_sign) {
    const int q = blockIdx.x;
    const int k = q % kPaths, i = (q / kPaths) % cin, o = q / (kPaths * cin);
    const int spb = kPtcThreads / m;
    const int r = threadIdx.x % m;
    const int64_t slen = 4 * NC * (int64_t)m;
    const int64_t field = 2 * g.vh * slen;
    double2 acc[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) acc[e] = make_double2(0.0, 0.0);
    if ((int)threadIdx.x < spb * m) {
        for (int64_t site = threadIdx.x / m; site < 2 * g.vh; site += spb) {
            float2 tv[4][NC], gv[4][NC];
            ptc_transport<NC>(tv, in + i * field + r, gauge, g, site, k, t_sign, m);
            const float2* gp = gout + o * field + site * slen + r;
#pragma unroll
            for (int s = 0; s < 4; ++s)
#pragma unroll
                for (int c = 0; c < NC; ++c) gv[s][c] = gp[(s * NC + c) * m];
#pragma unroll
            for (int sp = 0; sp < 4; ++sp)
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    float2 a = make_float2(0.f, 0.f);
#pragma unroll
                    for (int c = 0; c < NC; ++c)
                        a = cfma(gv[sp][c], make_float2(tv[s][c].x, -tv[s][c].y), a);
                    acc[sp * 4 + s].x += a.x;
                    acc[sp * 4 + s].y += a.y;
                }
        }
    }
    __shared__ double2 red[kPtcThreads / 32][16];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        double x = acc[e].x, y = acc[e].y;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            x += __shfl_down_sync(0xffffffffu, x, off);
            y += __shfl_down_sync(0xffffffffu, y, off);
        }
        if (lane == 0) red[warp][e] = make_double2(x, y);
    }
    __syncthreads();
    if (threadIdx.x < 16) {
        double2 s = make_double2(0.0, 0.0);
        for (int wi = 0; wi < kPtcThreads / 32; ++wi) {
            s.x += red[wi][threadIdx.x].x;
            s.y += red[wi][threadIdx.x].y;
        }
        gw[(int64_t)q * 16 + threadIdx.x] = s;
    }
}

__device__ __forceinline__ int opposite_path(int k) { return k == 0 ? 0 : (((k - 1) & 1) ? k - 1 : k + 1); }

// wadj[i][o][-k] = W[o][i][k]^dag (spin conjugate transpose): the adjoint layer
__global__ void ptc_adjoint_weights_kernel(float2* __restrict__ wadj, const float2* __restrict__ w, int cin,
                                           int cout) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= cout * cin * kPaths * 16) return;
    const int s = e & 3, sp = (e >> 2) & 3;
    const int k = (e >> 4) % kPaths;
    const int i = (e / (16 * kPaths)) % cin;
    const int o = e / (16 * kPaths * cin);
    const float2 v = w[e];
    wadj[(((int64_t)i * cout + o) * kPaths + opposite_path(k)) * 16 + s * 4 + sp] = make_float2(v.x, -v.y);
}

// Adam on the real and imaginary parts; the gradient of the real loss with respect to
// (Re w, Im w) is 2 gw.
__global__ void adam_kernel(float2* __restrict__ w, float2* __restrict__ m1, float2* __restrict__ m2,
                            const double2* __restrict__ gw, int64_t n, float lr, float b1, float b2, float eps,
                            float c1, float c2) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const float gx = (float)(2.0 * gw[e].x), gy = (float)(2.0 * gw[e].y);
    float2 a = m1[e], b = m2[e], x = w[e];
    a.x = b1 * a.x + (1.f - b1) * gx;
    a.y = b1 * a.y + (1.f - b1) * gy;
    b.x = b2 * b.x + (1.f - b2) * gx * gx;
    b.y = b2 * b.y + (1.f - b2) * gy * gy;
    x.x -= lr * (a.x / c1) / (sqrtf(b.x / c2) + eps);
    x.y -= lr * (a.y / c1) / (sqrtf(b.y / c2) + eps);
    m1[e] = a;
    m2[e] = b;
    w[e] = x;
}

__global__ void sub_kernel(float2* __restrict__ r, const float2* __restrict__ b, int64_t n) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        r[e].x -= b[e].x;
        r[e].y -= b[e].y;
    }
}

// g_j *= 1 / ||b_j||^2 (bnorm holds ||b_j||)
__global__ void scale_rhs_kernel(float2* __restrict__ g, const double* __restrict__ bnorm, int64_t n, int m) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const double bn = bnorm[e % m];
        const float s = bn > 0.0 ? (float)(1.0 / (bn * bn)) : 0.f;
        g[e].x *= s;
        g[e].y *= s;
    }
}

template <typename D, typename S>
__global__ void pc_cast_kernel(D* __restrict__ dst, const S* __restrict__ src, int64_t n, const int* __restrict__ done) {
    if (done != nullptr && *done) return;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const S v = src[e];
        dst[e].x = v.x;
        dst[e].y = v.y;
    }
}

// ---- FP64 BiCGStab reductions of the preconditioned solve ----
__global__ void __launch_bounds__(kRedThreads)
pc_alpha_kernel(const double2* __restrict__ r0, const double2* __restrict__ v, const BicgScalars* __restrict__ sc,
                int64_t n, int m, RedArgs ra) {
    if (sc->done) return;
    double2 acc[1] = {make_double2(0.0, 0.0)};
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const double2 a = r0[e], b = v[e];
        acc[0].x += a.x * b.x + a.y * b.y;
        acc[0].y += a.x * b.y - a.y * b.x;
    }
    grid_reduce<1>(acc, m, ra);
}

__global__ void __launch_bounds__(kRedThreads)
pc_omega_kernel(const double2* __restrict__ t, const double2* __restrict__ s, const BicgScalars* __restrict__ sc,
                int64_t n, int m, RedArgs ra) {
    if (sc->done) return;
    double2 acc[2] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const double2 a = t[e], b = s[e];
        acc[0].x += a.x * b.x + a.y * b.y;
        acc[0].y += a.x * b.y - a.y * b.x;
        acc[1].x += a.x * a.x + a.y * a.y;
    }
    grid_reduce<2>(acc, m, ra);
}

__global__ void __launch_bounds__(kRedThreads)
pc_xr_kernel(double2* __restrict__ x, double2* __restrict__ r, const double2* __restrict__ ph,
             const double2* __restrict__ sh, const double2* __restrict__ s, const double2* __restrict__ t,
             const double2* __restrict__ r0, const BicgScalars* __restrict__ sc, int64_t n, int m, RedArgs ra) {
    if (sc->done) return;
    const int j = threadIdx.x % m;
    const double2 al = sc->alpha[j], om = sc->omega[j];
    double2 acc[2] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const double2 a = ph[e], b = sh[e], sv = s[e], tv = t[e];
        double2 xv = x[e];
        xv.x += al.x * a.x - al.y * a.y + om.x * b.x - om.y * b.y;
        xv.y += al.x * a.y + al.y * a.x + om.x * b.y + om.y * b.x;
        x[e] = xv;
        const double2 rv = make_double2(sv.x - (om.x * tv.x - om.y * tv.y), sv.y - (om.x * tv.y + om.y * tv.x));
        r[e] = rv;
        const double2 q = r0[e];
        acc[0].x += rv.x * rv.x + rv.y * rv.y;
        acc[1].x += q.x * rv.x + q.y * rv.y;
        acc[1].y += q.x * rv.y - q.y * rv.x;
    }
    grid_reduce<2>(acc, m, ra);
}

int elem_grid(int64_t n) {
    const int64_t want = (n + 255) / 256;
    const int64_t cap = (int64_t)sm_count() * 8;
    return (int)(want < cap ? (want > 0 ? want : 1) : cap);
}

template <typename K>
int red_grid(K k, int block, int64_t n, const Scratch& ws) {
    int grid = resident_grid(k, block, n);
    return grid > ws.max_blocks ? ws.max_blocks : grid;
}

template <int NC>
int layer_launch(float2* out, const float2* in, const float2* w, const float2* gauge, const Geom& g, int m, int cin,
                 int cout, float t_sign, const int* done, cudaStream_t st) {
    const size_t smem = (size_t)cout * cin * kPaths * 16 * sizeof(float2);
    if (smem > 200 * 1024) return set_error(QCU_ERR_UNSUPPORTED, "layer weights exceed shared memory");
    const int per = m * cout;
    const int block = per <= kPtcThreads ? (kPtcThreads / per) * per : per;
    if (block > 1024) return set_error(QCU_ERR_UNSUPPORTED, "m_rhs * channels = %d > 1024", per);
    const int spb = block / per;
    const int64_t want = (2 * g.vh + spb - 1) / spb;
    const int64_t cap = (int64_t)sm_count() * 8;
    const int grid = (int)(want < cap ? want : cap);
    ptc_layer_kernel<NC><<<grid, block, smem, st>>>(out, in, w, gauge, g, m, cin, cout, t_sign, done);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

template <int NC>
int wgrad_launch(double2* gw, const float2* gout, const float2* in, const float2* gauge, const Geom& g, int m,
                 int cin, int cout, float t_sign, cudaStream_t st) {
    ptc_wgrad_kernel<NC><<<cout * cin * kPaths, kPtcThreads, 0, st>>>(gw, gout, in, gauge, g, m, cin, cout, t_sign);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

// raise the dynamic shared memory limit of the layer kernels (weights of one layer);
// done once at set-up, outside any stream capture
int ptc_set_attributes() {
    const int bytes = 200 * 1024;
    QCUB_CUDA_CHECK(cudaFuncSetAttribute(ptc_layer_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    QCUB_CUDA_CHECK(cudaFuncSetAttribute(ptc_layer_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    QCUB_CUDA_CHECK(cudaFuncSetAttribute(ptc_layer_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    return QCU_SUCCESS;
}

int layer(int nc, float2* out, const float2* in, const float2* w, const float2* gauge, const Geom& g, int m, int cin,
          int cout, float t_sign, const int* done, cudaStream_t st) {
    switch (nc) {
        case 2: return layer_launch<2>(out, in, w, gauge, g, m, cin, cout, t_sign, done, st);
        case 3: return layer_launch<3>(out, in, w, gauge, g, m, cin, cout, t_sign, done, st);
        case 4: return layer_launch<4>(out, in, w, gauge, g, m, cin, cout, t_sign, done, st);
        default: return set_error(QCU_ERR_UNSUPPORTED, "preconditioner n_color=%d (2..4)", nc);
    }
}

int wgrad(int nc, double2* gw, const float2* gout, const float2* in, const float2* gauge, const Geom& g, int m,
          int cin, int cout, float t_sign, cudaStream_t st) {
    switch (nc) {
        case 2: return wgrad_launch<2>(gw, gout, in, gauge, g, m, cin, cout, t_sign, st);
        case 3: return wgrad_launch<3>(gw, gout, in, gauge, g, m, cin, cout, t_sign, st);
        case 4: return wgrad_launch<4>(gw, gout, in, gauge, g, m, cin, cout, t_sign, st);
        default: return set_error(QCU_ERR_UNSUPPORTED, "preconditioner n_color=%d (2..4)", nc);
    }
}

}  // namespace

// ---------------- FP64 pieces of the preconditioned solve ----------------

int pc_alpha(const void* r0, const void* v, BicgScalars* sc, int64_t len, int m, const Scratch& ws, cudaStream_t st) {
    const int block = rhs_block(m);
    const int grid = red_grid(pc_alpha_kernel, block, len * m, ws);
    RedArgs ra{ws.partials, ws.counter, ws.result, sc, nullptr, FIN_ALPHA};
    pc_alpha_kernel<<<grid, block, 0, st>>>(static_cast<const double2*>(r0), static_cast<const double2*>(v), sc,
                                            len * m, m, ra);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

int pc_omega(const void* t, const void* s, BicgScalars* sc, int64_t len, int m, const Scratch& ws, cudaStream_t st) {
    const int block = rhs_block(m);
    const int grid = red_grid(pc_omega_kernel, block, len * m, ws);
    RedArgs ra{ws.partials, ws.counter, ws.result, sc, nullptr, FIN_OMEGA};
    pc_omega_kernel<<<grid, block, 0, st>>>(static_cast<const double2*>(t), static_cast<const double2*>(s), sc,
                                            len * m, m, ra);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

int pc_xr(void* x, void* r, const void* ph, const void* sh, const void* s, const void* t, const void* r0,
          BicgScalars* sc, int64_t len, int m, const Scratch& ws, cudaStream_t st) {
    const int block = rhs_block(m);
    const int grid = red_grid(pc_xr_kernel, block, len * m, ws);
    RedArgs ra{ws.partials, ws.counter, ws.result, sc, nullptr, FIN_BETA};
    pc_xr_kernel<<<grid, block, 0, st>>>(static_cast<double2*>(x), static_cast<double2*>(r),
                                         static_cast<const double2*>(ph), static_cast<const double2*>(sh),
                                         static_cast<const double2*>(s), static_cast<const double2*>(t),
                                         static_cast<const double2*>(r0), sc, len * m, m, ra);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

int pc_cast(void* dst, int dprec, const void* src, int sprec, int64_t n, const int* done, cudaStream_t st) {
    const int grid = elem_grid(n);
    if (dprec == QCU_PRECISION_SINGLE && sprec == QCU_PRECISION_DOUBLE)
        pc_cast_kernel<float2, double2><<<grid, 256, 0, st>>>(static_cast<float2*>(dst),
                                                              static_cast<const double2*>(src), n, done);
    else if (dprec == QCU_PRECISION_DOUBLE && sprec == QCU_PRECISION_SINGLE)
        pc_cast_kernel<double2, float2><<<grid, 256, 0, st>>>(static_cast<double2*>(dst),
                                                              static_cast<const float2*>(src), n, done);
    else
        return set_error(QCU_ERR_UNSUPPORTED, "preconditioner cast %d -> %d", sprec, dprec);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

int full_mat(void* out, const void* in, const void* gauge, const Geom& g, int nc, int m, double kappa,
             double t_sign, bool dagger, int prec, cudaStream_t st, const int* done) {
    const size_t hb = (size_t)g.vh * 4 * nc * m * 2 * prec_bytes(prec);
    for (int par = 0; par < 2; ++par) {
        HopParams p{};
        p.out = static_cast<char*>(out) + par * hb;
        p.in = static_cast<const char*>(in) + (1 - par) * hb;
        p.x = static_cast<const char*>(in) + par * hb;
        p.a = -kappa;
        p.gauge = gauge;
        p.g = g;
        p.m = m;
        p.parity = par;
        p.t_sign = t_sign;
        p.done = done;
        const int rc = hop_launch(p, nc, prec, dagger, EPI_XPAY, st);
        if (rc) return rc;
    }
    return QCU_SUCCESS;
}

// ---------------- Precond ----------------

int Precond::init(const int L[4], int n_color, int m_rhs, int n_layers, int channels, double t_boundary) {
    if (L[0] < 2 || L[0] % 2 || L[1] < 1 || L[2] < 1 || L[3] < 1)
        return set_error(QCU_ERR_INVALID, "lattice %dx%dx%dx%d (Lx must be even)", L[0], L[1], L[2], L[3]);
    if (n_color < 2 || n_color > 4) return set_error(QCU_ERR_UNSUPPORTED, "preconditioner n_color=%d (2..4)", n_color);
    if (m_rhs < 1 || m_rhs > kMaxRhs) return set_error(QCU_ERR_INVALID, "m_rhs=%d (1..%d)", m_rhs, kMaxRhs);
    if (n_layers < 1 || n_layers > 16) return set_error(QCU_ERR_INVALID, "layers=%d (1..16)", n_layers);
    if (channels < 1 || channels > 16 || (n_layers == 1 && channels != 1))
        return set_error(QCU_ERR_INVALID, "channels=%d (1..16; 1 for a single layer)", channels);
    if (m_rhs * channels > 1024) return set_error(QCU_ERR_UNSUPPORTED, "m_rhs * channels > 1024");
    if ((size_t)channels * channels * kPaths * 16 * sizeof(float2) > 200 * 1024)
        return set_error(QCU_ERR_UNSUPPORTED, "channels=%d: one layer's weights exceed shared memory", channels);
    if (t_boundary != 1.0 && t_boundary != -1.0) return set_error(QCU_ERR_INVALID, "t_boundary must be +1 or -1");
    g = make_geom(L);
    nc = n_color;
    m = m_rhs;
    layers = n_layers;
    ch = channels;
    t_sign = t_boundary;
    nw = 0;
    for (int l = 0; l < layers; ++l) {
        cin.push_back(l == 0 ? 1 : ch);
        cout.push_back(l == layers - 1 ? 1 : ch);
        woff.push_back(nw);
        nw += (int64_t)cout[l] * cin[l] * kPaths * 16;
    }
    int rc;
    if ((rc = ptc_set_attributes())) return rc;
    if ((rc = w.ensure(nw * sizeof(float2))) || (rc = wadj.ensure(nw * sizeof(float2))) ||
        (rc = gw.ensure(nw * sizeof(double2))) || (rc = m1.ensure(nw * sizeof(float2))) ||
        (rc = m2.ensure(nw * sizeof(float2))))
        return rc;
    const int nfields = 1 + ch * (layers - 1) + 1;
    if ((rc = act.ensure(nfields * field_bytes()))) return rc;
    for (auto& b : gbuf)
        if ((rc = b.ensure(ch * field_bytes()))) return rc;
    for (auto& b : tmp)
        if ((rc = b.ensure(field_bytes()))) return rc;
    if ((rc = norms.ensure(2 * kMaxRhs * sizeof(double)))) return rc;
    if ((rc = gauge.ensure((size_t)8 * g.vh * nc * nc * sizeof(float2)))) return rc;
    if (cudaMallocHost(&host_norms, 2 * kMaxRhs * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return set_error(QCU_ERR_ALLOC, "pinned host allocation failed");
    }
    if ((rc = scratch_alloc(&ws))) return rc;
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return set_error(QCU_ERR_CUDA, "stream creation failed");
    }
    QCUB_CUDA_CHECK(cudaMemsetAsync(w.ptr, 0, nw * sizeof(float2), stream));
    QCUB_CUDA_CHECK(cudaMemsetAsync(m1.ptr, 0, nw * sizeof(float2), stream));
    QCUB_CUDA_CHECK(cudaMemsetAsync(m2.ptr, 0, nw * sizeof(float2), stream));
    QCUB_CUDA_CHECK(cudaStreamSynchronize(stream));
    return QCU_SUCCESS;
}

void Precond::release() {
    if (stream) cudaStreamSynchronize(stream);
    scratch_free(&ws);
    if (host_norms) cudaFreeHost(host_norms);
    host_norms = nullptr;
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
}

int Precond::apply(float2* out, const float2* in, const void* gauge32, cudaStream_t st, const int* done) {
    const float2* gp = static_cast<const float2*>(gauge32);
    const float2* wp = static_cast<const float2*>(w.ptr);
    float2* fields = static_cast<float2*>(act.ptr);
    const int64_t fl = field_len();
    const float2* src = in;
    for (int l = 0; l < layers; ++l) {
        float2* dst = (l == layers - 1) ? out : fields + (int64_t)act_offset(l + 1) * fl;
        const int rc = layer(nc, dst, src, wp + woff[l], gp, g, m, cin[l], cout[l], (float)t_sign, done, st);
        if (rc) return rc;
        src = dst;
    }
    return QCU_SUCCESS;
}

int Precond::loss_grad(const float2* b, double kappa, double* loss, cudaStream_t st) {
    if (!has_gauge) return set_error(QCU_ERR_STATE, "preconditioner gauge field not set");
    const float2* gp = static_cast<const float2*>(gauge.ptr);
    const float2* wp = static_cast<const float2*>(w.ptr);
    float2* fields = static_cast<float2*>(act.ptr);
    const int64_t fl = field_len();
    const int64_t len = fl / m;   // complex per RHS
    int rc;
    // forward, keeping every layer's input
    QCUB_CUDA_CHECK(cudaMemcpyAsync(fields, b, field_bytes(), cudaMemcpyDeviceToDevice, st));
    for (int l = 0; l < layers; ++l) {
        if ((rc = layer(nc, fields + (int64_t)act_offset(l + 1) * fl, fields + (int64_t)act_offset(l) * fl,
                        wp + woff[l], gp, g, m, cin[l], cout[l], (float)t_sign, nullptr, st)))
            return rc;
    }
    const float2* y = fields + (int64_t)act_offset(layers) * fl;
    float2* r = static_cast<float2*>(tmp[0].ptr);
    float2* seed = static_cast<float2*>(gbuf[0].ptr);
    // r = M y - b ; seed = M^dag r / ||b||^2
    if ((rc = full_mat(r, y, gp, g, nc, m, kappa, t_sign, false, QCU_PRECISION_SINGLE, st))) return rc;
    sub_kernel<<<elem_grid(fl), 256, 0, st>>>(r, fields, fl);
    QCUB_CHECK_LAUNCH();
    double* dn = static_cast<double*>(norms.ptr);
    if ((rc = mrhs_norm(dn, r, len, m, QCU_PRECISION_SINGLE, ws, st))) return rc;
    if ((rc = mrhs_norm(dn + kMaxRhs, fields, len, m, QCU_PRECISION_SINGLE, ws, st))) return rc;
    if ((rc = full_mat(seed, r, gp, g, nc, m, kappa, t_sign, true, QCU_PRECISION_SINGLE, st))) return rc;
    scale_rhs_kernel<<<elem_grid(fl), 256, 0, st>>>(seed, dn + kMaxRhs, fl, m);
    QCUB_CHECK_LAUNCH();
    // backward
    int cur = 0;
    for (int l = layers - 1; l >= 0; --l) {
        const float2* gout = static_cast<const float2*>(gbuf[cur].ptr);
        if ((rc = wgrad(nc, static_cast<double2*>(gw.ptr) + woff[l], gout, fields + (int64_t)act_offset(l) * fl, gp, g,
                        m, cin[l], cout[l], (float)t_sign, st)))
            return rc;
        if (l == 0) break;
        const int nwl = cout[l] * cin[l] * kPaths * 16;
        float2* wa = static_cast<float2*>(wadj.ptr) + woff[l];
        ptc_adjoint_weights_kernel<<<(nwl + 255) / 256, 256, 0, st>>>(wa, wp + woff[l], cin[l], cout[l]);
        QCUB_CHECK_LAUNCH();
        if ((rc = layer(nc, static_cast<float2*>(gbuf[1 - cur].ptr), gout, wa, gp, g, m, cout[l], cin[l],
                        (float)t_sign, nullptr, st)))
            return rc;
        cur = 1 - cur;
    }
    QCUB_CUDA_CHECK(cudaMemcpyAsync(host_norms, dn, 2 * kMaxRhs * sizeof(double), cudaMemcpyDeviceToHost, st));
    QCUB_CUDA_CHECK(cudaStreamSynchronize(st));
    double l2 = 0.0;
    for (int j = 0; j < m; ++j) {
        const double bn = host_norms[kMaxRhs + j];
        if (bn > 0) l2 += (host_norms[j] * host_norms[j]) / (bn * bn);
    }
    if (loss) *loss = l2;
    return QCU_SUCCESS;
}

int Precond::adam(double lr, cudaStream_t st) {
    ++step;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
    adam_kernel<<<(int)((nw + 255) / 256), 256, 0, st>>>(static_cast<float2*>(w.ptr), static_cast<float2*>(m1.ptr),
                                                         static_cast<float2*>(m2.ptr),
                                                         static_cast<const double2*>(gw.ptr), nw, (float)lr, b1, b2,
                                                         1e-8f, c1, c2);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

}  // namespace qcub

using namespace qcub;

namespace {
Precond* as_precond(void* h) { return static_cast<Precond*>(h); }

// caller field (FP32 or FP64, gathered full lattice) -> FP32 field of the handle
int to_single(Precond& P, const void* src, int prec, float2* dst, cudaStream_t st) {
    if (prec == QCU_PRECISION_SINGLE) {
        QCUB_CUDA_CHECK(cudaMemcpyAsync(dst, src, P.field_bytes(), cudaMemcpyDeviceToDevice, st));
        return QCU_SUCCESS;
    }
    if (prec != QCU_PRECISION_DOUBLE) return set_error(QCU_ERR_UNSUPPORTED, "precision %d (single or double)", prec);
    return pc_cast(dst, QCU_PRECISION_SINGLE, src, QCU_PRECISION_DOUBLE, P.field_len(), nullptr, st);
}
}  // namespace

extern "C" {

int qcuPrecondCreate(void** handle, const int L[4], int n_color, int m_rhs, int layers, int channels,
                     double t_boundary) {
    clear_error();
    if (!handle || !L) return set_error(QCU_ERR_INVALID, "null pointer");
    *handle = nullptr;
    Precond* P = new Precond();
    const int rc = P->init(L, n_color, m_rhs, layers, channels, t_boundary);
    if (rc) {
        P->release();
        delete P;
        return rc;
    }
    *handle = P;
    return QCU_SUCCESS;
}

int qcuPrecondDestroy(void* handle) {
    clear_error();
    if (!handle) return QCU_SUCCESS;
    Precond* P = as_precond(handle);
    P->release();
    delete P;
    return QCU_SUCCESS;
}

int64_t qcuPrecondNumWeights(void* handle) {
    clear_error();
    if (!handle) return -set_error(QCU_ERR_INVALID, "null handle");
    return as_precond(handle)->nw;
}

int qcuPrecondSetWeights(void* handle, const float* weights) {
    clear_error();
    if (!handle || !weights) return set_error(QCU_ERR_INVALID, "null pointer");
    Precond& P = *as_precond(handle);
    QCUB_CUDA_CHECK(cudaMemcpyAsync(P.w.ptr, weights, P.nw * sizeof(float2), cudaMemcpyHostToDevice, P.stream));
    QCUB_CUDA_CHECK(cudaMemsetAsync(P.m1.ptr, 0, P.nw * sizeof(float2), P.stream));
    QCUB_CUDA_CHECK(cudaMemsetAsync(P.m2.ptr, 0, P.nw * sizeof(float2), P.stream));
    QCUB_CUDA_CHECK(cudaStreamSynchronize(P.stream));
    P.step = 0;
    return QCU_SUCCESS;
}

int qcuPrecondGetWeights(void* handle, float* weights) {
    clear_error();
    if (!handle || !weights) return set_error(QCU_ERR_INVALID, "null pointer");
    Precond& P = *as_precond(handle);
    QCUB_CUDA_CHECK(cudaMemcpyAsync(weights, P.w.ptr, P.nw * sizeof(float2), cudaMemcpyDeviceToHost, P.stream));
    QCUB_CUDA_CHECK(cudaStreamSynchronize(P.stream));
    return QCU_SUCCESS;
}

int qcuPrecondSetGauge(void* handle, const void* gauge, int precision) {
    clear_error();
    if (!handle || !gauge) return set_error(QCU_ERR_INVALID, "null pointer");
    Precond& P = *as_precond(handle);
    int rc = cast_complex(P.gauge.ptr, QCU_PRECISION_SINGLE, gauge, precision, 8 * P.g.vh * P.nc * P.nc, P.stream);
    if (rc) return rc;
    QCUB_CUDA_CHECK(cudaStreamSynchronize(P.stream));
    P.has_gauge = true;
    return QCU_SUCCESS;
}

int qcuPrecondApply(void* handle, void* out, const void* in, int precision, void* stream) {
    clear_error();
    if (!handle || !out || !in) return set_error(QCU_ERR_INVALID, "null pointer");
    Precond& P = *as_precond(handle);
    if (!P.has_gauge) return set_error(QCU_ERR_STATE, "preconditioner gauge field not set");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    float2* a = static_cast<float2*>(P.tmp[1].ptr);
    float2* b = static_cast<float2*>(P.tmp[2].ptr);
    int rc;
    if ((rc = to_single(P, in, precision, a, st))) return rc;
    if ((rc = P.apply(b, a, P.gauge.ptr, st))) return rc;
    if (precision == QCU_PRECISION_SINGLE) {
        QCUB_CUDA_CHECK(cudaMemcpyAsync(out, b, P.field_bytes(), cudaMemcpyDeviceToDevice, st));
    } else {
        if ((rc = pc_cast(out, QCU_PRECISION_DOUBLE, b, QCU_PRECISION_SINGLE, P.field_len(), nullptr, st))) return rc;
    }
    return QCU_SUCCESS;
}

int qcuPrecondLossGrad(void* handle, const void* b, int precision, double kappa, double* loss, double* grad) {
    clear_error();
    if (!handle || !b) return set_error(QCU_ERR_INVALID, "null pointer");
    Precond& P = *as_precond(handle);
    float2* bf = static_cast<float2*>(P.tmp[1].ptr);
    int rc;
    if ((rc = to_single(P, b, precision, bf, P.stream))) return rc;
    if ((rc = P.loss_grad(bf, kappa, loss, P.stream))) return rc;
    if (grad) {
        QCUB_CUDA_CHECK(cudaMemcpyAsync(grad, P.gw.ptr, P.nw * sizeof(double2), cudaMemcpyDeviceToHost, P.stream));
        QCUB_CUDA_CHECK(cudaStreamSynchronize(P.stream));
        for (int64_t e = 0; e < 2 * P.nw; ++e) grad[e] *= 2.0;   // d loss / d(Re w, Im w)
    }
    return QCU_SUCCESS;
}

int qcuPrecondTrainStep(void* handle, const void* b, int precision, double kappa, double lr, double* loss) {
    clear_error();
    if (!handle || !b) return set_error(QCU_ERR_INVALID, "null pointer");
    if (!(lr > 0)) return set_error(QCU_ERR_INVALID, "learning rate %g", lr);
    Precond& P = *as_precond(handle);
    float2* bf = static_cast<float2*>(P.tmp[1].ptr);
    int rc;
    if ((rc = to_single(P, b, precision, bf, P.stream))) return rc;
    if ((rc = P.loss_grad(bf, kappa, loss, P.stream))) return rc;
    if ((rc = P.adam(lr, P.stream))) return rc;
    QCUB_CUDA_CHECK(cudaStreamSynchronize(P.stream));
    return QCU_SUCCESS;
}

}  // extern "C"
