// dslash_impl.cuh -- multi-RHS Wilson hop term D_p on the gathered layout, SIMT.
//
// Operator (reference include/kernel/su_n_m_rhs_dslash.cuh:92-105 with the
// projector tables of include/kernel/complex_matmul.cuh:16-227, 503-600):
//   out(x) = sum_mu  U_mu(x) (1 - s g_mu) in(x + mu) + U_mu(x - mu)^dag (1 + s g_mu) in(x - mu)
// with s = +1, or s = -1 when the dagger flag is set; g_mu in the DeGrand-Rossi basis.
// Hops that cross the t boundary are multiplied by t_sign (+1 periodic as in the
// reference, -1 antiperiodic).
//
// Layout: in/out [Vh][4][N][m] complex (RHS fastest), gauge [4][2][Vh][N][N].
// Neighbour rule of include/point/qcu_point.cuh:16-61 (x moves only when the
// full-lattice x parity allows it; all directions wrap periodically).
//
// Work split: one thread per (half-site, RHS).  The block size is a multiple of m,
// so the m threads of a site are consecutive and read consecutive addresses of each
// (spin, colour) row; the N x N link of a site is read by its m threads and served
// from L1.  Each thread projects the neighbour's 4-spinor to two half spinors, applies
// the link (or its adjoint), and reconstructs into 4N complex accumulators.
#pragma once

#include "common.cuh"
#include "reduce.cuh"

namespace qcub {

enum HopEpilogue : int {
    EPI_PLAIN = 0,     // out = D in
    EPI_XPAY = 1,      // out = x + a * D in                      (a real)
    EPI_SCHUR_R0 = 2,  // out = x - a * D in;  reduce <r0, out>
    EPI_SCHUR_TS = 3,  // out = x - a * D in;  reduce <out, x>, <out, out>
    EPI_SCHUR = 4,     // out = x - a * D in;  no reduction
    EPI_RESID = 5,     // out = y - (x - a * D in), y = r0 pointer;  reduce |out|^2
};

struct HopParams {
    void* out;
    const void* in;
    const void* gauge;
    const void* x;     // epilogue vector (same layout and precision as out)
    const void* r0;    // epilogue dot partner
    Geom g;
    int m;
    int parity;        // output parity
    double t_sign;
    double a;
    RedArgs red;
    const int* done;   // if non-null and *done != 0 the kernel returns at once
    const int* gate;   // if non-null and *gate == 0 the kernel returns at once
    int blocked;       // 1: in, out, x and r0 in the site-blocked layout (kSiteBlock)
    // optional per-site tables (hop_tables.cu), read by the tensor-core hop when both are set:
    // hop-link array in the storage precision built for this t_sign, and neighbour table
    const void* links;
    const uint32_t* nbr;
    // optional per-RHS flags (device int[m]): the tensor-core hop skips every group of 4 RHS
    // whose flags are all 0 (its outputs are then left as they were); null = all active
    const int* active;
    // bounded waits of the staged tensor-core hop: the limit in clock cycles (0: about a
    // second), and a self-test mode in which its stages are armed but never filled, so that
    // every wait runs out and the kernel ends with the device error flag set
    long long wait_limit;
    int wait_test;
};

__device__ __forceinline__ bool skip_launch(const int* done, const int* gate) {
    return (done != nullptr && *done) || (gate != nullptr && !*gate);
}

template <typename A2, typename A>
__device__ __forceinline__ A2 scale2(A2 v, A f) {
    v.x *= f;
    v.y *= f;
    return v;
}

// One hop: project, multiply by the link, reconstruct into acc.
// MU: direction (0..3 = x,y,z,t); FWD: forward neighbour; SIG: sign of gamma in the projector.
template <int NC, typename S, int MU, bool FWD, int SIG>
__device__ __forceinline__ void hop_one(typename St<S>::A2 (&acc)[4][NC],
                                        const typename St<S>::S2* __restrict__ psi, int m,
                                        const typename St<S>::S2* __restrict__ U,
                                        typename St<S>::A fac) {
    using A2 = typename St<S>::A2;
    using A = typename St<S>::A;
    constexpr A sg = (A)SIG;
    A2 h0[NC], h1[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const A2 p0 = St<S>::ld(psi[(0 * NC + c) * m]);
        const A2 p1 = St<S>::ld(psi[(1 * NC + c) * m]);
        const A2 p2 = St<S>::ld(psi[(2 * NC + c) * m]);
        const A2 p3 = St<S>::ld(psi[(3 * NC + c) * m]);
        if (MU == 0) {        // h0 = p0 + s i p3 ; h1 = p1 + s i p2
            h0[c] = mk2<A2>(p0.x - sg * p3.y, p0.y + sg * p3.x);
            h1[c] = mk2<A2>(p1.x - sg * p2.y, p1.y + sg * p2.x);
        } else if (MU == 1) { // h0 = p0 - s p3 ; h1 = p1 + s p2
            h0[c] = mk2<A2>(p0.x - sg * p3.x, p0.y - sg * p3.y);
            h1[c] = mk2<A2>(p1.x + sg * p2.x, p1.y + sg * p2.y);
        } else if (MU == 2) { // h0 = p0 + s i p2 ; h1 = p1 - s i p3
            h0[c] = mk2<A2>(p0.x - sg * p2.y, p0.y + sg * p2.x);
            h1[c] = mk2<A2>(p1.x + sg * p3.y, p1.y - sg * p3.x);
        } else {              // h0 = p0 + s p2 ; h1 = p1 + s p3
            h0[c] = mk2<A2>(p0.x + sg * p2.x, p0.y + sg * p2.y);
            h1[c] = mk2<A2>(p1.x + sg * p3.x, p1.y + sg * p3.y);
        }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        A2 w0 = mk2<A2>(0, 0), w1 = mk2<A2>(0, 0);
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            if (FWD) {
                const A2 u = St<S>::ld(U[c * NC + k]);
                cmac(w0, u, h0[k]);
                cmac(w1, u, h1[k]);
            } else {
                const A2 u = St<S>::ld(U[k * NC + c]);
                cmac_conj(w0, u, h0[k]);
                cmac_conj(w1, u, h1[k]);
            }
        }
        if (MU == 3) {
            w0 = scale2(w0, fac);
            w1 = scale2(w1, fac);
        }
        acc[0][c].x += w0.x; acc[0][c].y += w0.y;
        acc[1][c].x += w1.x; acc[1][c].y += w1.y;
        if (MU == 0) {        // acc2 += -s i w1 ; acc3 += -s i w0
            acc[2][c].x += sg * w1.y; acc[2][c].y -= sg * w1.x;
            acc[3][c].x += sg * w0.y; acc[3][c].y -= sg * w0.x;
        } else if (MU == 1) { // acc2 += s w1 ; acc3 += -s w0
            acc[2][c].x += sg * w1.x; acc[2][c].y += sg * w1.y;
            acc[3][c].x -= sg * w0.x; acc[3][c].y -= sg * w0.y;
        } else if (MU == 2) { // acc2 += -s i w0 ; acc3 += s i w1
            acc[2][c].x += sg * w0.y; acc[2][c].y -= sg * w0.x;
            acc[3][c].x -= sg * w1.y; acc[3][c].y += sg * w1.x;
        } else {              // acc2 += s w0 ; acc3 += s w1
            acc[2][c].x += sg * w0.x; acc[2][c].y += sg * w0.y;
            acc[3][c].x += sg * w1.x; acc[3][c].y += sg * w1.y;
        }
    }
}

// Gather the 8 hops of one (site, rhs) into acc.
template <int NC, typename S, bool DAG>
__device__ __forceinline__ void hop_site(typename St<S>::A2 (&acc)[4][NC], const HopParams& p,
                                         int64_t site, int rhs) {
    using S2 = typename St<S>::S2;
    using A = typename St<S>::A;
    using A2 = typename St<S>::A2;
    const S2* __restrict__ in = static_cast<const S2*>(p.in);
    const S2* __restrict__ gauge = static_cast<const S2*>(p.gauge);
    const int lxh = p.g.lxh, Ly = p.g.L[1], Lz = p.g.L[2], Lt = p.g.L[3];
    const int64_t vh = p.g.vh;
    const int parity = p.parity;
    const int m = p.m;
    // half-site coordinates
    const SiteXYZT sc = site_coords(p.g, (uint32_t)site);
    const int xh = sc.xh, y = sc.y, z = sc.z, t = sc.t;
    const int xodd = (parity ^ (y + z + t)) & 1;  // full x = 2 xh + xodd
    const int64_t sy = lxh, sz = (int64_t)lxh * Ly, st = sz * Lz;
    const int64_t site_len = (int64_t)kNs * NC * m;
    constexpr int N2 = NC * NC;
    // forward sign s_f = -s, backward s_b = +s  (s = +1, or -1 with dagger)
    constexpr int SF = DAG ? 1 : -1;
    constexpr int SB = DAG ? -1 : 1;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[i][c] = mk2<A2>(0, 0);

    const S2* gf = gauge + (int64_t)parity * vh * N2;        // + mu*2*vh*N2
    const S2* gb = gauge + (int64_t)(1 - parity) * vh * N2;
    const int64_t gmu = 2 * vh * N2;

    // ---- x ----
    {
        const int64_t nf = site - xh + (xodd ? (xh + 1 == lxh ? 0 : xh + 1) : xh);
        hop_one<NC, S, 0, true, SF>(acc, in + nf * site_len + rhs, m, gf + site * N2, (A)1);
        const int64_t nb = site - xh + (xodd ? xh : (xh == 0 ? lxh - 1 : xh - 1));
        hop_one<NC, S, 0, false, SB>(acc, in + nb * site_len + rhs, m, gb + nb * N2, (A)1);
    }
    // ---- y ----
    {
        const int64_t nf = site + (y + 1 == Ly ? -(int64_t)(Ly - 1) * sy : sy);
        hop_one<NC, S, 1, true, SF>(acc, in + nf * site_len + rhs, m, gf + gmu + site * N2, (A)1);
        const int64_t nb = site + (y == 0 ? (int64_t)(Ly - 1) * sy : -sy);
        hop_one<NC, S, 1, false, SB>(acc, in + nb * site_len + rhs, m, gb + gmu + nb * N2, (A)1);
    }
    // ---- z ----
    {
        const int64_t nf = site + (z + 1 == Lz ? -(int64_t)(Lz - 1) * sz : sz);
        hop_one<NC, S, 2, true, SF>(acc, in + nf * site_len + rhs, m, gf + 2 * gmu + site * N2, (A)1);
        const int64_t nb = site + (z == 0 ? (int64_t)(Lz - 1) * sz : -sz);
        hop_one<NC, S, 2, false, SB>(acc, in + nb * site_len + rhs, m, gb + 2 * gmu + nb * N2, (A)1);
    }
    // ---- t ----
    {
        const bool wf = (t + 1 == Lt);
        const int64_t nf = site + (wf ? -(int64_t)(Lt - 1) * st : st);
        hop_one<NC, S, 3, true, SF>(acc, in + nf * site_len + rhs, m, gf + 3 * gmu + site * N2,
                                    wf ? (A)p.t_sign : (A)1);
        const bool wb = (t == 0);
        const int64_t nb = site + (wb ? (int64_t)(Lt - 1) * st : -st);
        hop_one<NC, S, 3, false, SB>(acc, in + nb * site_len + rhs, m, gb + 3 * gmu + nb * N2,
                                     wb ? (A)p.t_sign : (A)1);
    }
}

// Epilogue of one (site, RHS): store out = D in (EPI_PLAIN) or the fused combination
// with x / r0, and add this thread's terms of the fused reductions to red.
// `base` is the offset of (site, spin 0, colour 0, RHS) in the gathered layout.
template <int NC, typename S, int EPI, int NV>
__device__ __forceinline__ void hop_store(const typename St<S>::A2 (&acc)[4][NC], const HopParams& p,
                                          int64_t base, typename St<S>::A2 (&red)[NV > 0 ? NV : 1]) {
    using S2 = typename St<S>::S2;
    using A = typename St<S>::A;
    using A2 = typename St<S>::A2;
    const int m = p.m;
    S2* __restrict__ out = static_cast<S2*>(p.out);
    const S2* __restrict__ xv = static_cast<const S2*>(p.x);
    const S2* __restrict__ r0 = static_cast<const S2*>(p.r0);
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const int64_t o = base + (int64_t)(s * NC + c) * m;
            A2 v = acc[s][c];
            if (EPI == EPI_PLAIN) {
                out[o] = St<S>::cv(v);
            } else {
                const A2 xx = St<S>::ld(xv[o]);
                const A a = (A)p.a;
                A2 res;
                if (EPI == EPI_XPAY) {
                    res = mk2<A2>(xx.x + a * v.x, xx.y + a * v.y);
                } else if (EPI == EPI_RESID) {
                    const A2 yy = St<S>::ld(r0[o]);
                    res = mk2<A2>(yy.x - xx.x + a * v.x, yy.y - xx.y + a * v.y);
                } else {
                    res = mk2<A2>(xx.x - a * v.x, xx.y - a * v.y);
                }
                const S2 rs = St<S>::cv(res);
                out[o] = rs;
                if (NV > 0) {
                    // per-thread partial sums in the arithmetic type (FP64 for FP64 storage,
                    // FP32 otherwise); the sums across threads and blocks are FP64
                    const A2 rr = St<S>::ld(rs);
                    if (EPI == EPI_RESID) {
                        red[0].x += rr.x * rr.x + rr.y * rr.y;
                    } else if (EPI == EPI_SCHUR_R0) {   // <r0, out> = sum conj(r0) out
                        const A2 q = St<S>::ld(r0[o]);
                        red[0].x += q.x * rr.x + q.y * rr.y;
                        red[0].y += q.x * rr.y - q.y * rr.x;
                    } else if (EPI == EPI_SCHUR_TS) {  // <out, x>, <out, out>
                        red[0].x += rr.x * xx.x + rr.y * xx.y;
                        red[0].y += rr.x * xx.y - rr.y * xx.x;
                        red[NV - 1].x += rr.x * rr.x + rr.y * rr.y;
                    }
                }
            }
        }
}

// Minimum resident blocks per SM requested from the register allocator: FP64 at small N
// otherwise takes ~190 registers (one block per SM, latency-bound); capping it at 128
// doubles the warps in flight.  Large N keeps the compiler's choice (accumulators dominate).
template <int NC, typename S>
struct HopMinBlocks {
    static constexpr int value = NC <= 4 ? (sizeof(S) == 8 ? 2 : 3) : 1;
};

template <int NC, typename S, bool DAG, int EPI>
__global__ void __launch_bounds__(kRedThreads, HopMinBlocks<NC, S>::value) hop_kernel(const HopParams p) {
    using S2 = typename St<S>::S2;
    using A = typename St<S>::A;
    using A2 = typename St<S>::A2;
    constexpr int NV = (EPI == EPI_SCHUR_R0 || EPI == EPI_RESID) ? 1 : (EPI == EPI_SCHUR_TS ? 2 : 0);
    if (skip_launch(p.done, p.gate)) return;
    const int m = p.m;
    const int rhs = threadIdx.x % m;
    const int64_t total = p.g.vh * m;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t site_len = (int64_t)kNs * NC * m;
    A2 red[NV > 0 ? NV : 1];
#pragma unroll
    for (int k = 0; k < (NV > 0 ? NV : 1); ++k) red[k] = mk2<A2>(0, 0);

    // block size and grid stride are multiples of m: the thread keeps RHS tid % m and
    // walks sites without dividing
    const int64_t site_stride = stride / m;
    (void)total;
    for (int64_t site = ((int64_t)blockIdx.x * blockDim.x) / m + threadIdx.x / m; site < p.g.vh;
         site += site_stride) {
        A2 acc[4][NC];
        hop_site<NC, S, DAG>(acc, p, site, rhs);
        hop_store<NC, S, EPI, NV>(acc, p, site * site_len + rhs, red);
    }
    if constexpr (NV > 0) {
        double2 rv[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) rv[k] = make_double2((double)red[k].x, (double)red[k].y);
        grid_reduce<NV>(rv, m, p.red);
    }
}

// ---------------------------------------------------------------------------------
// Colour-split variant: one thread per (half-site, RHS, output colour c).  The thread
// projects the full neighbour spinor (the N threads of one (site, RHS) are adjacent
// lanes and read the same addresses, which the load unit merges), applies row c of
// the link (column c of its adjoint), and keeps only 4 complex accumulators.  This
// trades more load/projection instructions for far fewer registers: it lifts
// occupancy for FP64 and makes large N (6, 8) fit without spilling.
// Block size and grid stride are multiples of N*m; thread tid works on
// c = tid % N, RHS = (tid / N) % m.
template <int NC, typename S, bool DAG, int EPI>
__global__ void __launch_bounds__(kRedThreads) hop_kernel_cs(const HopParams p) {
    using S2 = typename St<S>::S2;
    using A = typename St<S>::A;
    using A2 = typename St<S>::A2;
    constexpr int NV = (EPI == EPI_SCHUR_R0 || EPI == EPI_RESID) ? 1 : (EPI == EPI_SCHUR_TS ? 2 : 0);
    constexpr int SF = DAG ? 1 : -1;    // sign of gamma in the forward projector
    constexpr int SB = DAG ? -1 : 1;    // ... in the backward projector
    constexpr int N2 = NC * NC;
    if (skip_launch(p.done, p.gate)) return;
    const int m = p.m;
    const int c = threadIdx.x % NC;
    const int rhs = (threadIdx.x / NC) % m;
    const int64_t per_site = (int64_t)NC * m;
    const int64_t site_stride = ((int64_t)gridDim.x * blockDim.x) / per_site;
    const int64_t site_len = (int64_t)kNs * NC * m;
    const S2* __restrict__ in = static_cast<const S2*>(p.in);
    const S2* __restrict__ gauge = static_cast<const S2*>(p.gauge);
    S2* __restrict__ out = static_cast<S2*>(p.out);
    const S2* __restrict__ xv = static_cast<const S2*>(p.x);
    const S2* __restrict__ r0 = static_cast<const S2*>(p.r0);
    const int lxh = p.g.lxh, Ly = p.g.L[1], Lz = p.g.L[2], Lt = p.g.L[3];
    const int64_t vh = p.g.vh;
    const int64_t sy = lxh, sz = (int64_t)lxh * Ly, st = sz * Lz;
    const int parity = p.parity;
    const S2* gf = gauge + (int64_t)parity * vh * N2;
    const S2* gb = gauge + (int64_t)(1 - parity) * vh * N2;
    const int64_t gmu = 2 * vh * N2;
    double2 red[NV > 0 ? NV : 1];
#pragma unroll
    for (int k = 0; k < (NV > 0 ? NV : 1); ++k) red[k] = make_double2(0.0, 0.0);

    for (int64_t site = ((int64_t)blockIdx.x * blockDim.x) / per_site + threadIdx.x / per_site; site < vh;
         site += site_stride) {
        const SiteXYZT sc = site_coords(p.g, (uint32_t)site);
        const int xh = sc.xh, y = sc.y, z = sc.z, t = sc.t;
        const int xodd = (parity ^ (y + z + t)) & 1;
        A2 acc[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[i] = mk2<A2>(0, 0);
#pragma unroll
        for (int h = 0; h < 8; ++h) {
            const int mu = h >> 1;
            const bool fwd = (h & 1) == 0;
            int64_t nb;
            bool wrap = false;
            if (mu == 0) {
                nb = fwd ? site - xh + (xodd ? (xh + 1 == lxh ? 0 : xh + 1) : xh)
                         : site - xh + (xodd ? xh : (xh == 0 ? lxh - 1 : xh - 1));
            } else if (mu == 1) {
                nb = fwd ? site + (y + 1 == Ly ? -(int64_t)(Ly - 1) * sy : sy)
                         : site + (y == 0 ? (int64_t)(Ly - 1) * sy : -sy);
            } else if (mu == 2) {
                nb = fwd ? site + (z + 1 == Lz ? -(int64_t)(Lz - 1) * sz : sz)
                         : site + (z == 0 ? (int64_t)(Lz - 1) * sz : -sz);
            } else {
                wrap = fwd ? (t + 1 == Lt) : (t == 0);
                nb = fwd ? site + (wrap ? -(int64_t)(Lt - 1) * st : st)
                         : site + (wrap ? (int64_t)(Lt - 1) * st : -st);
            }
            const A sg = (A)(fwd ? SF : SB);
            const S2* psi = in + nb * site_len + rhs;
            const S2* U = fwd ? gf + mu * gmu + site * N2 : gb + mu * gmu + nb * N2;
            A2 w0 = mk2<A2>(0, 0), w1 = mk2<A2>(0, 0);
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                const A2 p0 = St<S>::ld(psi[(0 * NC + k) * m]);
                const A2 p1 = St<S>::ld(psi[(1 * NC + k) * m]);
                const A2 p2 = St<S>::ld(psi[(2 * NC + k) * m]);
                const A2 p3 = St<S>::ld(psi[(3 * NC + k) * m]);
                A2 h0, h1;
                if (mu == 0) {
                    h0 = mk2<A2>(p0.x - sg * p3.y, p0.y + sg * p3.x);
                    h1 = mk2<A2>(p1.x - sg * p2.y, p1.y + sg * p2.x);
                } else if (mu == 1) {
                    h0 = mk2<A2>(p0.x - sg * p3.x, p0.y - sg * p3.y);
                    h1 = mk2<A2>(p1.x + sg * p2.x, p1.y + sg * p2.y);
                } else if (mu == 2) {
                    h0 = mk2<A2>(p0.x - sg * p2.y, p0.y + sg * p2.x);
                    h1 = mk2<A2>(p1.x + sg * p3.y, p1.y - sg * p3.x);
                } else {
                    h0 = mk2<A2>(p0.x + sg * p2.x, p0.y + sg * p2.y);
                    h1 = mk2<A2>(p1.x + sg * p3.x, p1.y + sg * p3.y);
                }
                if (fwd) {
                    const A2 u = St<S>::ld(U[c * NC + k]);
                    cmac(w0, u, h0);
                    cmac(w1, u, h1);
                } else {
                    const A2 u = St<S>::ld(U[k * NC + c]);
                    cmac_conj(w0, u, h0);
                    cmac_conj(w1, u, h1);
                }
            }
            if (wrap) {
                w0 = scale2(w0, (A)p.t_sign);
                w1 = scale2(w1, (A)p.t_sign);
            }
            acc[0].x += w0.x; acc[0].y += w0.y;
            acc[1].x += w1.x; acc[1].y += w1.y;
            if (mu == 0) {
                acc[2].x += sg * w1.y; acc[2].y -= sg * w1.x;
                acc[3].x += sg * w0.y; acc[3].y -= sg * w0.x;
            } else if (mu == 1) {
                acc[2].x += sg * w1.x; acc[2].y += sg * w1.y;
                acc[3].x -= sg * w0.x; acc[3].y -= sg * w0.y;
            } else if (mu == 2) {
                acc[2].x += sg * w0.y; acc[2].y -= sg * w0.x;
                acc[3].x -= sg * w1.y; acc[3].y += sg * w1.x;
            } else {
                acc[2].x += sg * w0.x; acc[2].y += sg * w0.y;
                acc[3].x += sg * w1.x; acc[3].y += sg * w1.y;
            }
        }
        const int64_t base = site * site_len + rhs + (int64_t)c * m;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int64_t o = base + (int64_t)s * NC * m;
            const A2 v = acc[s];
            if (EPI == EPI_PLAIN) {
                out[o] = St<S>::cv(v);
            } else {
                const A2 xx = St<S>::ld(xv[o]);
                const A a = (A)p.a;
                A2 res;
                if (EPI == EPI_XPAY) {
                    res = mk2<A2>(xx.x + a * v.x, xx.y + a * v.y);
                } else if (EPI == EPI_RESID) {
                    const A2 yy = St<S>::ld(r0[o]);
                    res = mk2<A2>(yy.x - xx.x + a * v.x, yy.y - xx.y + a * v.y);
                } else {
                    res = mk2<A2>(xx.x - a * v.x, xx.y - a * v.y);
                }
                const S2 rs = St<S>::cv(res);
                out[o] = rs;
                if (NV > 0) {
                    const A2 rr = St<S>::ld(rs);
                    if (EPI == EPI_RESID) {
                        red[0].x += (double)rr.x * rr.x + (double)rr.y * rr.y;
                    } else if (EPI == EPI_SCHUR_R0) {
                        const A2 q = St<S>::ld(r0[o]);
                        red[0].x += (double)q.x * rr.x + (double)q.y * rr.y;
                        red[0].y += (double)q.x * rr.y - (double)q.y * rr.x;
                    } else if (EPI == EPI_SCHUR_TS) {
                        red[0].x += (double)rr.x * xx.x + (double)rr.y * xx.y;
                        red[0].y += (double)rr.x * xx.y - (double)rr.y * xx.x;
                        red[NV - 1].x += (double)rr.x * rr.x + (double)rr.y * rr.y;
                    }
                }
            }
        }
    }
    if constexpr (NV > 0) {
        double2 rv[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) rv[k] = red[k];
        grid_reduce<NV>(rv, m, p.red, NC);
    }
}

// Host launcher for one instantiation (defined in the per-precision .cu files).
template <int NC, typename S>
int launch_hop(const HopParams& p, bool dagger, int epi, cudaStream_t stream, bool color_split);

}  // namespace qcub
