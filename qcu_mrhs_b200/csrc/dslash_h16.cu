// dslash_h16.cu -- multi-RHS hop term for FP16 / BF16 storage in packed 16-bit arithmetic.
//
// Same operator, layouts and epilogues as dslash_impl.cuh (reference
// include/kernel/su_n_m_rhs_dslash.cuh:92-105, complex_matmul.cuh:16-600).  What differs:
//   * the 8 links of every site are read once per block, not once per (site, RHS)
//     thread: a staging pass writes each link element W = U (forward) or U^dag
//     (backward, with the t-boundary sign folded in) to shared memory as the pair of
//     packed words (W.re, W.im), (-W.im, W.re), and the 8 neighbour indices next to it;
//   * the spin projection and the link products run on packed complex numbers
//     (one half2 / bfloat162 word = re, im): W h = (h.re, h.re) * (W.re, W.im)
//                                               + (h.im, h.im) * (-W.im, W.re),
//     two packed FMAs per complex multiply-add and no conversions;
//   * each hop's result is converted to FP32 and accumulated over the 8 hops in FP32
//     (ACC16 = false), or accumulated in the storage format (ACC16 = true, as the
//     reference's half-precision wmma path does).
// One thread per (half-site, RHS); the m threads of a site are consecutive.
#include <type_traits>

#include "dslash.h"
#include "dslash_impl.cuh"
#include "workspace.h"

namespace qcub {

namespace {

template <typename S> struct Pk16;
template <> struct Pk16<__half> {
    using T2 = __half2;
    __device__ static T2 fma(T2 a, T2 b, T2 c) { return __hfma2(a, b, c); }
    __device__ static T2 add(T2 a, T2 b) { return __hadd2(a, b); }
    __device__ static T2 sub(T2 a, T2 b) { return __hsub2(a, b); }
    __device__ static float2 f32(T2 v) { return __half22float2(v); }
};
template <> struct Pk16<__nv_bfloat16> {
    using T2 = __nv_bfloat162;
    __device__ static T2 fma(T2 a, T2 b, T2 c) { return __hfma2(a, b, c); }
    __device__ static T2 add(T2 a, T2 b) { return __hadd2(a, b); }
    __device__ static T2 sub(T2 a, T2 b) { return __hsub2(a, b); }
    __device__ static float2 f32(T2 v) { return __bfloat1622float2(v); }
};

template <typename T2>
__device__ __forceinline__ uint32_t bits(T2 v) { return *reinterpret_cast<uint32_t*>(&v); }
template <typename T2>
__device__ __forceinline__ T2 word(uint32_t u) { return *reinterpret_cast<T2*>(&u); }

// packed-word helpers (re in the low half, im in the high half; sign bit 15 / 31)
__device__ __forceinline__ uint32_t times_i(uint32_t u) { return __byte_perm(u, 0, 0x1032) ^ 0x00008000u; }   // i v
__device__ __forceinline__ uint32_t times_mi(uint32_t u) { return __byte_perm(u, 0, 0x1032) ^ 0x80000000u; }  // -i v
__device__ __forceinline__ uint32_t bcast_re(uint32_t u) { return __byte_perm(u, 0, 0x1010); }
__device__ __forceinline__ uint32_t bcast_im(uint32_t u) { return __byte_perm(u, 0, 0x3232); }
// the same broadcasts through the half-pair intrinsics, which the compiler can fold into
// the operand selection of the packed FMA that consumes them (no separate instruction)
template <typename T2> __device__ __forceinline__ T2 lo2(uint32_t u);
template <typename T2> __device__ __forceinline__ T2 hi2(uint32_t u);
template <> __device__ __forceinline__ __half2 lo2<__half2>(uint32_t u) { return __low2half2(word<__half2>(u)); }
template <> __device__ __forceinline__ __half2 hi2<__half2>(uint32_t u) { return __high2half2(word<__half2>(u)); }
template <> __device__ __forceinline__ __nv_bfloat162 lo2<__nv_bfloat162>(uint32_t u) {
    return __low2bfloat162(word<__nv_bfloat162>(u));
}
template <> __device__ __forceinline__ __nv_bfloat162 hi2<__nv_bfloat162>(uint32_t u) {
    return __high2bfloat162(word<__nv_bfloat162>(u));
}

constexpr int kH16Threads = 256;
constexpr int kH16MaxSites = 32;   // sites staged per block pass

template <int NC>
struct H16Smem {
    static constexpr int kStride = 8 * NC * NC + 1;   // uint2 per site, padded against bank conflicts
    uint2 link[kH16MaxSites * kStride];
    int nb[kH16MaxSites][8];
};

// half index of the neighbour of `site` (parity `parity`) along hop h = 2 mu + (backward)
__device__ __forceinline__ int64_t h16_neighbour(const Geom& g, int64_t site, int parity, int h, bool* wrap) {
    const SiteXYZT c = site_coords(g, (uint32_t)site);
    const int lxh = g.lxh, Ly = g.L[1], Lz = g.L[2], Lt = g.L[3];
    const int64_t sy = lxh, sz = (int64_t)lxh * Ly, st = sz * Lz;
    const int mu = h >> 1;
    const bool f = (h & 1) == 0;
    *wrap = false;
    if (mu == 0) {
        const int xodd = (parity ^ (c.y + c.z + c.t)) & 1;
        return f ? site - c.xh + (xodd ? (c.xh + 1 == lxh ? 0 : c.xh + 1) : c.xh)
                 : site - c.xh + (xodd ? c.xh : (c.xh == 0 ? lxh - 1 : c.xh - 1));
    }
    if (mu == 1) return f ? site + (c.y + 1 == Ly ? -(int64_t)(Ly - 1) * sy : sy) : site + (c.y == 0 ? (int64_t)(Ly - 1) * sy : -sy);
    if (mu == 2) return f ? site + (c.z + 1 == Lz ? -(int64_t)(Lz - 1) * sz : sz) : site + (c.z == 0 ? (int64_t)(Lz - 1) * sz : -sz);
    *wrap = f ? (c.t + 1 == Lt) : (c.t == 0);
    return f ? site + (*wrap ? -(int64_t)(Lt - 1) * st : st) : site + (*wrap ? (int64_t)(Lt - 1) * st : -st);
}

// One hop of one (site, RHS): project the neighbour spinor, multiply by the staged link,
// reconstruct into acc.  SG: sign s of gamma in this hop's projector (1 - s g or 1 + s g).
template <int NC, typename S, bool ACC16, int MU, int SG, typename AccT, typename LinkFn>
__device__ __forceinline__ void h16_hop(AccT (&acc)[4][NC], const uint32_t* __restrict__ psi, int m,
                                        LinkFn link) {
    using P = Pk16<S>;
    using T2 = typename P::T2;
    uint32_t h0[NC], h1[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const uint32_t p0 = __ldg(psi + (0 * NC + c) * m);
        const uint32_t p1 = __ldg(psi + (1 * NC + c) * m);
        const uint32_t p2 = __ldg(psi + (2 * NC + c) * m);
        const uint32_t p3 = __ldg(psi + (3 * NC + c) * m);
        if (MU == 0) {        // h0 = p0 + s i p3 ; h1 = p1 + s i p2
            h0[c] = bits(P::add(word<T2>(p0), word<T2>(SG > 0 ? times_i(p3) : times_mi(p3))));
            h1[c] = bits(P::add(word<T2>(p1), word<T2>(SG > 0 ? times_i(p2) : times_mi(p2))));
        } else if (MU == 1) { // h0 = p0 - s p3 ; h1 = p1 + s p2
            h0[c] = bits(SG > 0 ? P::sub(word<T2>(p0), word<T2>(p3)) : P::add(word<T2>(p0), word<T2>(p3)));
            h1[c] = bits(SG > 0 ? P::add(word<T2>(p1), word<T2>(p2)) : P::sub(word<T2>(p1), word<T2>(p2)));
        } else if (MU == 2) { // h0 = p0 + s i p2 ; h1 = p1 - s i p3
            h0[c] = bits(P::add(word<T2>(p0), word<T2>(SG > 0 ? times_i(p2) : times_mi(p2))));
            h1[c] = bits(P::add(word<T2>(p1), word<T2>(SG > 0 ? times_mi(p3) : times_i(p3))));
        } else {              // h0 = p0 + s p2 ; h1 = p1 + s p3
            h0[c] = bits(SG > 0 ? P::add(word<T2>(p0), word<T2>(p2)) : P::sub(word<T2>(p0), word<T2>(p2)));
            h1[c] = bits(SG > 0 ? P::add(word<T2>(p1), word<T2>(p3)) : P::sub(word<T2>(p1), word<T2>(p3)));
        }
    }
    uint32_t r0[NC], i0[NC], r1[NC], i1[NC];
#pragma unroll
    for (int k = 0; k < NC; ++k) {
        r0[k] = bcast_re(h0[k]);
        i0[k] = bcast_im(h0[k]);
        r1[k] = bcast_re(h1[k]);
        i1[k] = bcast_im(h1[k]);
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        T2 w0 = word<T2>(0u), w1 = word<T2>(0u);
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            const uint2 l = link(c, k);
            w0 = P::fma(word<T2>(r0[k]), word<T2>(l.x), w0);
            w0 = P::fma(word<T2>(i0[k]), word<T2>(l.y), w0);
            w1 = P::fma(word<T2>(r1[k]), word<T2>(l.x), w1);
            w1 = P::fma(word<T2>(i1[k]), word<T2>(l.y), w1);
        }
        // reconstruction: acc0 += w0, acc1 += w1, acc2/acc3 from the projector
        if constexpr (ACC16) {
            const uint32_t b0 = bits(w0), b1 = bits(w1);
            uint32_t a2, a3;   // terms added to spins 2 and 3
            if (MU == 0) {        // acc2 += -s i w1 ; acc3 += -s i w0
                a2 = SG > 0 ? times_mi(b1) : times_i(b1);
                a3 = SG > 0 ? times_mi(b0) : times_i(b0);
            } else if (MU == 1) { // acc2 += s w1 ; acc3 += -s w0
                a2 = SG > 0 ? b1 : b1 ^ 0x80008000u;
                a3 = SG > 0 ? b0 ^ 0x80008000u : b0;
            } else if (MU == 2) { // acc2 += -s i w0 ; acc3 += s i w1
                a2 = SG > 0 ? times_mi(b0) : times_i(b0);
                a3 = SG > 0 ? times_i(b1) : times_mi(b1);
            } else {              // acc2 += s w0 ; acc3 += s w1
                a2 = SG > 0 ? b0 : b0 ^ 0x80008000u;
                a3 = SG > 0 ? b1 : b1 ^ 0x80008000u;
            }
            acc[0][c] = P::add(acc[0][c], w0);
            acc[1][c] = P::add(acc[1][c], w1);
            acc[2][c] = P::add(acc[2][c], word<T2>(a2));
            acc[3][c] = P::add(acc[3][c], word<T2>(a3));
        } else {
            // convert the two products once; the +-i and sign of spins 2, 3 are free in FP32
            const float2 f0 = P::f32(w0), f1 = P::f32(w1);
            constexpr float sg = (float)SG;
            acc[0][c].x += f0.x; acc[0][c].y += f0.y;
            acc[1][c].x += f1.x; acc[1][c].y += f1.y;
            if (MU == 0) {        // -i w = (w.im, -w.re)
                acc[2][c].x += sg * f1.y; acc[2][c].y -= sg * f1.x;
                acc[3][c].x += sg * f0.y; acc[3][c].y -= sg * f0.x;
            } else if (MU == 1) {
                acc[2][c].x += sg * f1.x; acc[2][c].y += sg * f1.y;
                acc[3][c].x -= sg * f0.x; acc[3][c].y -= sg * f0.y;
            } else if (MU == 2) {
                acc[2][c].x += sg * f0.y; acc[2][c].y -= sg * f0.x;
                acc[3][c].x -= sg * f1.y; acc[3][c].y += sg * f1.x;
            } else {
                acc[2][c].x += sg * f0.x; acc[2][c].y += sg * f0.y;
                acc[3][c].x += sg * f1.x; acc[3][c].y += sg * f1.y;
            }
        }
    }
}

template <int NC, typename S, bool DAG, int EPI, bool ACC16>
__global__ void __launch_bounds__(kH16Threads, 3) hop16_kernel(const HopParams p) {
    using P = Pk16<S>;
    using T2 = typename P::T2;
    using AccT = typename std::conditional<ACC16, T2, float2>::type;
    constexpr int NV = (EPI == EPI_SCHUR_R0 || EPI == EPI_RESID) ? 1 : (EPI == EPI_SCHUR_TS ? 2 : 0);
    constexpr int N2 = NC * NC;
    constexpr int SF = DAG ? 1 : -1;   // forward projector 1 - s g: sign of gamma
    constexpr int SB = DAG ? -1 : 1;   // backward projector 1 + s g
    __shared__ H16Smem<NC> sm;
    if (skip_launch(p.done, p.gate)) return;
    const int m = p.m;
    const int spb = blockDim.x / m;
    const int64_t vh = p.g.vh;
    const int parity = p.parity;
    const int64_t site_len = (int64_t)kNs * NC * m;
    const uint32_t* __restrict__ in = static_cast<const uint32_t*>(p.in);
    const uint32_t* __restrict__ gauge = static_cast<const uint32_t*>(p.gauge);
    const uint32_t tflip = p.t_sign < 0 ? 0x80008000u : 0u;
    const int sl = threadIdx.x / m;
    const int rhs = threadIdx.x - sl * m;
    float2 red[NV > 0 ? NV : 1];   // per-thread partial sums (FP64 across threads and blocks)
#pragma unroll
    for (int k = 0; k < (NV > 0 ? NV : 1); ++k) red[k] = make_float2(0.f, 0.f);

    for (int64_t base = (int64_t)blockIdx.x * spb; base < vh; base += (int64_t)gridDim.x * spb) {
        __syncthreads();   // the previous pass has finished reading the staged links
        // neighbours of the block's sites (8 per site); the wrap flag rides in bit 31
        for (int e = threadIdx.x; e < spb * 8; e += blockDim.x) {
            const int s = e >> 3, h = e & 7;
            const int64_t site = base + s;
            if (site < vh) {
                bool wrap;
                const int64_t nb = h16_neighbour(p.g, site, parity, h, &wrap);
                sm.nb[s][h] = (int)nb | (wrap ? (int)0x80000000u : 0);
            }
        }
        __syncthreads();
        // links: W = U_mu(x) forward, U_mu(x - mu)^dag backward, t-wrap sign folded in
        for (int e = threadIdx.x; e < spb * 8 * N2; e += blockDim.x) {
            const int s = e / (8 * N2);
            const int rem = e - s * 8 * N2;
            const int h = rem / N2, el = rem - h * N2;
            const int c = el / NC, k = el - c * NC;
            const int64_t site = base + s;
            if (site >= vh) continue;
            const int mu = h >> 1;
            const int nbw = sm.nb[s][h];
            uint32_t w;
            if ((h & 1) == 0) {
                w = __ldg(gauge + ((int64_t)(mu * 2 + parity) * vh + site) * N2 + c * NC + k);
            } else {
                const int64_t nb = nbw & 0x7fffffff;
                w = __ldg(gauge + ((int64_t)(mu * 2 + (1 - parity)) * vh + nb) * N2 + k * NC + c) ^ 0x80000000u;
            }
            if (nbw < 0) w ^= tflip;
            sm.link[s * H16Smem<NC>::kStride + h * N2 + el] = make_uint2(w, times_i(w));
        }
        __syncthreads();
        const int64_t site = base + sl;
        if (sl < spb && site < vh) {
            AccT acc[4][NC];
#pragma unroll
            for (int s = 0; s < 4; ++s)
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    if constexpr (ACC16) acc[s][c] = word<T2>(0u);
                    else acc[s][c] = make_float2(0.f, 0.f);
                }
            const uint2* L = sm.link + sl * H16Smem<NC>::kStride;
            const int* nbs = sm.nb[sl];
            const uint32_t* src = in + rhs;
#define QCUB_H16_HOP(H, MU, SIGN)                                                                     \
    h16_hop<NC, S, ACC16, MU, SIGN>(acc, src + (int64_t)(nbs[H] & 0x7fffffff) * site_len, m,              \
                                    [&](int c, int k) { return L[(H) * N2 + c * NC + k]; })
            QCUB_H16_HOP(0, 0, SF);
            QCUB_H16_HOP(1, 0, SB);
            QCUB_H16_HOP(2, 1, SF);
            QCUB_H16_HOP(3, 1, SB);
            QCUB_H16_HOP(4, 2, SF);
            QCUB_H16_HOP(5, 2, SB);
            QCUB_H16_HOP(6, 3, SF);
            QCUB_H16_HOP(7, 3, SB);
#undef QCUB_H16_HOP
            float2 facc[4][NC];
#pragma unroll
            for (int s = 0; s < 4; ++s)
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    if constexpr (ACC16) facc[s][c] = P::f32(acc[s][c]);
                    else facc[s][c] = acc[s][c];
                }
            hop_store<NC, S, EPI, NV>(facc, p, site * site_len + rhs, red);
        }
    }
    if constexpr (NV > 0) {
        double2 rv[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) rv[k] = make_double2((double)red[k].x, (double)red[k].y);
        grid_reduce<NV>(rv, m, p.red);
    }
}

// Variant without shared-memory staging: every (site, RHS) thread reads the links
// itself (the m threads of a site read the same words) and forms (-W.im, W.re) in
// registers; no block synchronisation, so the loads of different sites overlap freely.
template <int NC, bool FWD>
__device__ __forceinline__ void h16_load_link(uint32_t (&w)[NC * NC], const uint32_t* __restrict__ U, uint32_t flip) {
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int k = 0; k < NC; ++k)
            w[c * NC + k] = FWD ? (__ldg(U + c * NC + k) ^ flip) : (__ldg(U + k * NC + c) ^ 0x80000000u ^ flip);
}

// MR > 0: the RHS count is the compile-time constant MR (p.m == MR), so every spinor
// offset (s N + c) m is an immediate of its load; MR = 0: runtime m.
template <int NC, typename S, bool DAG, int EPI, bool ACC16, int MR>
__global__ void __launch_bounds__(kH16Threads, 4) hop16d_kernel(const HopParams p) {
    using P = Pk16<S>;
    using T2 = typename P::T2;
    using AccT = typename std::conditional<ACC16, T2, float2>::type;
    constexpr int NV = (EPI == EPI_SCHUR_R0 || EPI == EPI_RESID) ? 1 : (EPI == EPI_SCHUR_TS ? 2 : 0);
    constexpr int N2 = NC * NC;
    constexpr int SF = DAG ? 1 : -1;
    constexpr int SB = DAG ? -1 : 1;
    if (skip_launch(p.done, p.gate)) return;
    const int m = MR > 0 ? MR : p.m;
    const int rhs = threadIdx.x % m;
    const int64_t vh = p.g.vh;
    const int parity = p.parity;
    const int64_t site_len = (int64_t)kNs * NC * m;
    const uint32_t* __restrict__ in = static_cast<const uint32_t*>(p.in) + rhs;
    const uint32_t* __restrict__ gauge = static_cast<const uint32_t*>(p.gauge);
    const uint32_t tflip = p.t_sign < 0 ? 0x80008000u : 0u;
    const int lxh = p.g.lxh, Ly = p.g.L[1], Lz = p.g.L[2], Lt = p.g.L[3];
    const int64_t sy = lxh, sz = (int64_t)lxh * Ly, st = sz * Lz;
    const uint32_t* gf = gauge + (int64_t)parity * vh * N2;
    const uint32_t* gb = gauge + (int64_t)(1 - parity) * vh * N2;
    const int64_t gmu = 2 * vh * N2;
    float2 red[NV > 0 ? NV : 1];   // per-thread partial sums (FP64 across threads and blocks)
#pragma unroll
    for (int k = 0; k < (NV > 0 ? NV : 1); ++k) red[k] = make_float2(0.f, 0.f);
    const int64_t site_stride = ((int64_t)gridDim.x * blockDim.x) / m;
    for (int64_t site = ((int64_t)blockIdx.x * blockDim.x) / m + threadIdx.x / m; site < vh; site += site_stride) {
        if constexpr (EPI != EPI_PLAIN) {
            // the epilogue operands of this site (a contiguous site_len-word block) are
            // fetched into L2 while the hops are computed: one 128-byte line per thread
            const int64_t off = (int64_t)rhs * 32;   // words
            if (off < site_len) {
                asm volatile("prefetch.global.L2 [%0];" ::"l"(static_cast<const uint32_t*>(p.x) + site * site_len + off));
                if (EPI == EPI_SCHUR_R0 || EPI == EPI_RESID)
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(static_cast<const uint32_t*>(p.r0) + site * site_len + off));
            }
        }
        const SiteXYZT c = site_coords(p.g, (uint32_t)site);
        const int xodd = (parity ^ (c.y + c.z + c.t)) & 1;
        AccT acc[4][NC];
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
            for (int cc = 0; cc < NC; ++cc) {
                if constexpr (ACC16) acc[s][cc] = word<T2>(0u);
                else acc[s][cc] = make_float2(0.f, 0.f);
            }
        uint32_t w[N2];
        auto link = [&](int a, int b) { return make_uint2(w[a * NC + b], times_i(w[a * NC + b])); };
        // x
        {
            const int64_t nf = site - c.xh + (xodd ? (c.xh + 1 == lxh ? 0 : c.xh + 1) : c.xh);
            h16_load_link<NC, true>(w, gf + site * N2, 0u);
            h16_hop<NC, S, ACC16, 0, SF>(acc, in + nf * site_len, m, link);
            const int64_t nb = site - c.xh + (xodd ? c.xh : (c.xh == 0 ? lxh - 1 : c.xh - 1));
            h16_load_link<NC, false>(w, gb + nb * N2, 0u);
            h16_hop<NC, S, ACC16, 0, SB>(acc, in + nb * site_len, m, link);
        }
        // y
        {
            const int64_t nf = site + (c.y + 1 == Ly ? -(int64_t)(Ly - 1) * sy : sy);
            h16_load_link<NC, true>(w, gf + gmu + site * N2, 0u);
            h16_hop<NC, S, ACC16, 1, SF>(acc, in + nf * site_len, m, link);
            const int64_t nb = site + (c.y == 0 ? (int64_t)(Ly - 1) * sy : -sy);
            h16_load_link<NC, false>(w, gb + gmu + nb * N2, 0u);
            h16_hop<NC, S, ACC16, 1, SB>(acc, in + nb * site_len, m, link);
        }
        // z
        {
            const int64_t nf = site + (c.z + 1 == Lz ? -(int64_t)(Lz - 1) * sz : sz);
            h16_load_link<NC, true>(w, gf + 2 * gmu + site * N2, 0u);
            h16_hop<NC, S, ACC16, 2, SF>(acc, in + nf * site_len, m, link);
            const int64_t nb = site + (c.z == 0 ? (int64_t)(Lz - 1) * sz : -sz);
            h16_load_link<NC, false>(w, gb + 2 * gmu + nb * N2, 0u);
            h16_hop<NC, S, ACC16, 2, SB>(acc, in + nb * site_len, m, link);
        }
        // t (the wrap sign is folded into the link)
        {
            const bool wf = (c.t + 1 == Lt);
            const int64_t nf = site + (wf ? -(int64_t)(Lt - 1) * st : st);
            h16_load_link<NC, true>(w, gf + 3 * gmu + site * N2, wf ? tflip : 0u);
            h16_hop<NC, S, ACC16, 3, SF>(acc, in + nf * site_len, m, link);
            const bool wb = (c.t == 0);
            const int64_t nb = site + (wb ? (int64_t)(Lt - 1) * st : -st);
            h16_load_link<NC, false>(w, gb + 3 * gmu + nb * N2, wb ? tflip : 0u);
            h16_hop<NC, S, ACC16, 3, SB>(acc, in + nb * site_len, m, link);
        }
        float2 facc[4][NC];
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
            for (int cc = 0; cc < NC; ++cc) {
                if constexpr (ACC16) facc[s][cc] = P::f32(acc[s][cc]);
                else facc[s][cc] = acc[s][cc];
            }
        if constexpr (MR > 0) {
            HopParams q = p;   // lets hop_store see the constant RHS count
            q.m = MR;
            hop_store<NC, S, EPI, NV>(facc, q, site * site_len + rhs, red);
        } else {
            hop_store<NC, S, EPI, NV>(facc, p, site * site_len + rhs, red);
        }
    }
    if constexpr (NV > 0) {
        double2 rv[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) rv[k] = make_double2((double)red[k].x, (double)red[k].y);
        grid_reduce<NV>(rv, m, p.red);
    }
}

template <int NC, typename S, bool ACC16, int MR>
int launch16d_m(const HopParams& p, bool dagger, int epi, cudaStream_t st) {
    if (dagger && epi != EPI_PLAIN && epi != EPI_XPAY)
        return set_error(QCU_ERR_UNSUPPORTED, "dagger hop only with plain/xpay epilogue");
    void (*k)(const HopParams) = nullptr;
    switch (epi) {
        case EPI_PLAIN: k = dagger ? hop16d_kernel<NC, S, true, EPI_PLAIN, ACC16, MR> : hop16d_kernel<NC, S, false, EPI_PLAIN, ACC16, MR>; break;
        case EPI_XPAY: k = dagger ? hop16d_kernel<NC, S, true, EPI_XPAY, ACC16, MR> : hop16d_kernel<NC, S, false, EPI_XPAY, ACC16, MR>; break;
        case EPI_SCHUR_R0: k = hop16d_kernel<NC, S, false, EPI_SCHUR_R0, ACC16, MR>; break;
        case EPI_SCHUR_TS: k = hop16d_kernel<NC, S, false, EPI_SCHUR_TS, ACC16, MR>; break;
        case EPI_SCHUR: k = hop16d_kernel<NC, S, false, EPI_SCHUR, ACC16, MR>; break;
        case EPI_RESID: k = hop16d_kernel<NC, S, false, EPI_RESID, ACC16, MR>; break;
        default: return set_error(QCU_ERR_INVALID, "epilogue %d", epi);
    }
    const int block = (kH16Threads / p.m) * p.m;
    int grid = resident_grid(k, block, p.g.vh * p.m);
    if (grid > kScratchBlocks) grid = kScratchBlocks;
    k<<<grid, block, 0, st>>>(p);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

// 8-byte asynchronous global -> shared copy (cp.async, completion by wait_group)
__device__ __forceinline__ void cp_async8(uint2* smem, const uint2* gmem) {
    const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(a), "l"(gmem) : "memory");
}

// packed FP32 pair arithmetic (add.rn.f32x2 / sub: sm_100): one instruction per complex add
__device__ __forceinline__ uint64_t f2_bits(float2 v) {
    return (uint64_t)__float_as_uint(v.x) | ((uint64_t)__float_as_uint(v.y) << 32);
}
__device__ __forceinline__ float2 f2_from(uint64_t u) {
    return make_float2(__uint_as_float((uint32_t)u), __uint_as_float((uint32_t)(u >> 32)));
}
__device__ __forceinline__ void f2_add(float2& a, float2 b) {
    uint64_t z;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(z) : "l"(f2_bits(a)), "l"(f2_bits(b)));
    a = f2_from(z);
}
__device__ __forceinline__ void f2_sub(float2& a, float2 b) {
    uint64_t z;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(z) : "l"(f2_bits(a)), "l"(f2_bits(b)));
    a = f2_from(z);
}

// ---- two RHS per thread (compile-time even m) ----
// Thread per (half-site, RHS pair j): RHS 2j and 2j+1 sit in one 8-byte word pair of every
// (spin, colour) row, so each neighbour value is one 8-byte load; the links, their
// (-W.im, W.re) partners and the neighbour arithmetic serve both RHS.  psi points at the
// neighbour's row 0 (plus the pair); rs is the distance between rows in 8-byte words
// (m / 2 in the gathered layout, kSiteBlock m / 2 in the site-blocked one).
template <int NC, typename S, int MU, int SG, typename LinkFn>
__device__ __forceinline__ void h16_hop2(float2 (&acc)[2][4][NC], const uint2* __restrict__ psi, int rs,
                                         LinkFn link) {
    using P = Pk16<S>;
    using T2 = typename P::T2;
    uint32_t h0[2][NC], h1[2][NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const uint2 q0 = __ldg(psi + (0 * NC + c) * rs);
        const uint2 q1 = __ldg(psi + (1 * NC + c) * rs);
        const uint2 q2 = __ldg(psi + (2 * NC + c) * rs);
        const uint2 q3 = __ldg(psi + (3 * NC + c) * rs);
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const uint32_t p0 = r ? q0.y : q0.x, p1 = r ? q1.y : q1.x;
            const uint32_t p2 = r ? q2.y : q2.x, p3 = r ? q3.y : q3.x;
            if (MU == 0) {
                h0[r][c] = bits(P::add(word<T2>(p0), word<T2>(SG > 0 ? times_i(p3) : times_mi(p3))));
                h1[r][c] = bits(P::add(word<T2>(p1), word<T2>(SG > 0 ? times_i(p2) : times_mi(p2))));
            } else if (MU == 1) {
                h0[r][c] = bits(SG > 0 ? P::sub(word<T2>(p0), word<T2>(p3)) : P::add(word<T2>(p0), word<T2>(p3)));
                h1[r][c] = bits(SG > 0 ? P::add(word<T2>(p1), word<T2>(p2)) : P::sub(word<T2>(p1), word<T2>(p2)));
            } else if (MU == 2) {
                h0[r][c] = bits(P::add(word<T2>(p0), word<T2>(SG > 0 ? times_i(p2) : times_mi(p2))));
                h1[r][c] = bits(P::add(word<T2>(p1), word<T2>(SG > 0 ? times_mi(p3) : times_i(p3))));
            } else {
                h0[r][c] = bits(SG > 0 ? P::add(word<T2>(p0), word<T2>(p2)) : P::sub(word<T2>(p0), word<T2>(p2)));
                h1[r][c] = bits(SG > 0 ? P::add(word<T2>(p1), word<T2>(p3)) : P::sub(word<T2>(p1), word<T2>(p3)));
            }
        }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        T2 w0[2] = {word<T2>(0u), word<T2>(0u)}, w1[2] = {word<T2>(0u), word<T2>(0u)};
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            const uint2 l = link(c, k);
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                w0[r] = P::fma(lo2<T2>(h0[r][k]), word<T2>(l.x), w0[r]);
                w0[r] = P::fma(hi2<T2>(h0[r][k]), word<T2>(l.y), w0[r]);
                w1[r] = P::fma(lo2<T2>(h1[r][k]), word<T2>(l.x), w1[r]);
                w1[r] = P::fma(hi2<T2>(h1[r][k]), word<T2>(l.y), w1[r]);
            }
        }
        constexpr float sg = (float)SG;
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const float2 f0 = P::f32(w0[r]), f1 = P::f32(w1[r]);
            float2 (&a)[4][NC] = acc[r];
            // spins 0, 1 and the real-coefficient terms of spins 2, 3 as packed pair adds;
            // the +-i terms swap re and im, which stays scalar
            f2_add(a[0][c], f0);
            f2_add(a[1][c], f1);
            if (MU == 0) {
                a[2][c].x += sg * f1.y; a[2][c].y -= sg * f1.x;
                a[3][c].x += sg * f0.y; a[3][c].y -= sg * f0.x;
            } else if (MU == 1) {
                if (SG > 0) { f2_add(a[2][c], f1); f2_sub(a[3][c], f0); }
                else { f2_sub(a[2][c], f1); f2_add(a[3][c], f0); }
            } else if (MU == 2) {
                a[2][c].x += sg * f0.y; a[2][c].y -= sg * f0.x;
                a[3][c].x -= sg * f1.y; a[3][c].y += sg * f1.x;
            } else {
                if (SG > 0) { f2_add(a[2][c], f0); f2_add(a[3][c], f1); }
                else { f2_sub(a[2][c], f0); f2_sub(a[3][c], f1); }
            }
        }
    }
}

// Block and grid reduction when thread t holds the partial sums of RHS 2 (t % (m/2)) and
// 2 (t % (m/2)) + 1: fixed summation order, then the common last-block finisher.
template <int NV>
__device__ inline void grid_reduce_pairs(const float2 (&v)[2][NV > 0 ? NV : 1], int m, const RedArgs& ra) {
    __shared__ double2 sh[NV][2][kH16Threads];
    __shared__ double2 bsum[NV * kMaxRhs];
    const int tid = threadIdx.x, nb = blockDim.x, half = m >> 1;
#pragma unroll
    for (int k = 0; k < NV; ++k)
#pragma unroll
        for (int q = 0; q < 2; ++q) sh[k][q][tid] = make_double2((double)v[q][k].x, (double)v[q][k].y);
    __syncthreads();
    for (int idx = tid; idx < NV * m; idx += nb) {
        const int k = idx / m, rhs = idx - k * m;
        const int j = rhs >> 1, q = rhs & 1;
        double2 s = make_double2(0.0, 0.0);
        for (int t = j; t < nb; t += half) {
            s.x += sh[k][q][t].x;
            s.y += sh[k][q][t].y;
        }
        bsum[idx] = s;
    }
    __syncthreads();
    publish_and_finish<NV>(bsum, m, ra);
}

template <int NC, typename S, bool DAG, int EPI, int MR, bool BLK>
__global__ void __launch_bounds__(kH16Threads, 2) hop16p_kernel(const HopParams p) {
    using P = Pk16<S>;
    using S2 = typename St<S>::S2;
    using A2 = typename St<S>::A2;
    constexpr int NV = (EPI == EPI_SCHUR_R0 || EPI == EPI_RESID) ? 1 : (EPI == EPI_SCHUR_TS ? 2 : 0);
    constexpr int N2 = NC * NC;
    constexpr int SF = DAG ? 1 : -1;
    constexpr int SB = DAG ? -1 : 1;
    constexpr int M2 = MR / 2;
    static_assert(MR % 2 == 0, "two RHS per thread need an even RHS count");
    if (skip_launch(p.done, p.gate)) return;
    const int j = threadIdx.x % M2;                // RHS pair
    const int64_t vh = p.g.vh;
    const int parity = p.parity;
    const uint2* __restrict__ in2 = reinterpret_cast<const uint2*>(p.in) + j;
    const uint32_t* __restrict__ gauge = static_cast<const uint32_t*>(p.gauge);
    const uint32_t tflip = p.t_sign < 0 ? 0x80008000u : 0u;
    const int lxh = p.g.lxh, Ly = p.g.L[1], Lz = p.g.L[2], Lt = p.g.L[3];
    const int64_t sy = lxh, sz = (int64_t)lxh * Ly, st = sz * Lz;
    const uint32_t* gf = gauge + (int64_t)parity * vh * N2;
    const uint32_t* gb = gauge + (int64_t)(1 - parity) * vh * N2;
    const int64_t gmu = 2 * vh * N2;
    float2 red[2][NV > 0 ? NV : 1];
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int k = 0; k < (NV > 0 ? NV : 1); ++k) red[q][k] = make_float2(0.f, 0.f);
    const int64_t site_stride = ((int64_t)gridDim.x * blockDim.x) / M2;
    // 8-byte word of (site n, row 0, pair 0) and the distance between rows
    constexpr int64_t RS = BLK ? (int64_t)kSiteBlock * M2 : M2;
    auto sbase = [](int64_t n) -> int64_t {
        if constexpr (BLK) return (n / kSiteBlock) * (kNs * NC * kSiteBlock * M2) + (n % kSiteBlock) * M2;
        else return n * (kNs * NC * M2);
    };
    // Epilogue operands (x, and r0 where the epilogue reads it) are copied into shared memory
    // with cp.async when a site starts, so the copies land while its 8 hops compute and hold
    // no registers.  Layout [operand][row][thread] in 8-byte words; every thread reads back
    // only the words it copied itself, so no block barrier is needed.
    constexpr int NX = EPI == EPI_PLAIN ? 0 : ((EPI == EPI_SCHUR_R0 || EPI == EPI_RESID) ? 2 : 1);
    extern __shared__ uint2 h16_epi[];
    const int nthr = blockDim.x;
    for (int64_t site = ((int64_t)blockIdx.x * blockDim.x) / M2 + threadIdx.x / M2; site < vh; site += site_stride) {
        if constexpr (NX > 0) {
            const int64_t b2 = sbase(site) + j;
#pragma unroll
            for (int r = 0; r < kNs * NC; ++r) {
                cp_async8(&h16_epi[r * nthr + threadIdx.x], reinterpret_cast<const uint2*>(p.x) + b2 + r * RS);
                if constexpr (NX == 2)
                    cp_async8(&h16_epi[(kNs * NC + r) * nthr + threadIdx.x],
                              reinterpret_cast<const uint2*>(p.r0) + b2 + r * RS);
            }
            asm volatile("cp.async.commit_group;" ::: "memory");
        }
        const SiteXYZT c = site_coords(p.g, (uint32_t)site);
        const int xodd = (parity ^ (c.y + c.z + c.t)) & 1;
        float2 acc[2][4][NC];
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
            for (int s = 0; s < 4; ++s)
#pragma unroll
                for (int cc = 0; cc < NC; ++cc) acc[r][s][cc] = make_float2(0.f, 0.f);
        uint32_t w[N2];
        auto link = [&](int a, int b) { return make_uint2(w[a * NC + b], times_i(w[a * NC + b])); };
        {
            const int64_t nf = site - c.xh + (xodd ? (c.xh + 1 == lxh ? 0 : c.xh + 1) : c.xh);
            h16_load_link<NC, true>(w, gf + site * N2, 0u);
            h16_hop2<NC, S, 0, SF>(acc, in2 + sbase(nf), RS, link);
            const int64_t nb = site - c.xh + (xodd ? c.xh : (c.xh == 0 ? lxh - 1 : c.xh - 1));
            h16_load_link<NC, false>(w, gb + nb * N2, 0u);
            h16_hop2<NC, S, 0, SB>(acc, in2 + sbase(nb), RS, link);
        }
        {
            const int64_t nf = site + (c.y + 1 == Ly ? -(int64_t)(Ly - 1) * sy : sy);
            h16_load_link<NC, true>(w, gf + gmu + site * N2, 0u);
            h16_hop2<NC, S, 1, SF>(acc, in2 + sbase(nf), RS, link);
            const int64_t nb = site + (c.y == 0 ? (int64_t)(Ly - 1) * sy : -sy);
            h16_load_link<NC, false>(w, gb + gmu + nb * N2, 0u);
            h16_hop2<NC, S, 1, SB>(acc, in2 + sbase(nb), RS, link);
        }
        {
            const int64_t nf = site + (c.z + 1 == Lz ? -(int64_t)(Lz - 1) * sz : sz);
            h16_load_link<NC, true>(w, gf + 2 * gmu + site * N2, 0u);
            h16_hop2<NC, S, 2, SF>(acc, in2 + sbase(nf), RS, link);
            const int64_t nb = site + (c.z == 0 ? (int64_t)(Lz - 1) * sz : -sz);
            h16_load_link<NC, false>(w, gb + 2 * gmu + nb * N2, 0u);
            h16_hop2<NC, S, 2, SB>(acc, in2 + sbase(nb), RS, link);
        }
        {
            const bool wf = (c.t + 1 == Lt);
            const int64_t nf = site + (wf ? -(int64_t)(Lt - 1) * st : st);
            h16_load_link<NC, true>(w, gf + 3 * gmu + site * N2, wf ? tflip : 0u);
            h16_hop2<NC, S, 3, SF>(acc, in2 + sbase(nf), RS, link);
            const bool wb = (c.t == 0);
            const int64_t nb = site + (wb ? (int64_t)(Lt - 1) * st : -st);
            h16_load_link<NC, false>(w, gb + 3 * gmu + nb * N2, wb ? tflip : 0u);
            h16_hop2<NC, S, 3, SB>(acc, in2 + sbase(nb), RS, link);
        }
        // epilogue: the two RHS of every (spin, colour) row as one 8-byte word pair
        uint2* __restrict__ out2 = reinterpret_cast<uint2*>(p.out);
        const int64_t base2 = sbase(site) + j;
        if constexpr (NX > 0) asm volatile("cp.async.wait_group 0;" ::: "memory");
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
            for (int cc = 0; cc < NC; ++cc) {
                const int64_t o = base2 + (int64_t)(s * NC + cc) * RS;
                if (EPI == EPI_PLAIN) {
                    const S2 a0 = St<S>::cv(acc[0][s][cc]), a1 = St<S>::cv(acc[1][s][cc]);
                    out2[o] = make_uint2(bits(a0), bits(a1));
                } else {
                    const uint2 xw = h16_epi[(s * NC + cc) * nthr + threadIdx.x];
                    uint2 yw = make_uint2(0u, 0u);
                    if (EPI == EPI_RESID || EPI == EPI_SCHUR_R0) yw = h16_epi[(kNs * NC + s * NC + cc) * nthr + threadIdx.x];
                    uint32_t res_bits[2];
#pragma unroll
                    for (int r = 0; r < 2; ++r) {
                        const A2 v = acc[r][s][cc];
                        const A2 xx = St<S>::ld(word<S2>(r ? xw.y : xw.x));
                        const float a = (float)p.a;
                        A2 res;
                        if (EPI == EPI_XPAY) {
                            res = mk2<A2>(xx.x + a * v.x, xx.y + a * v.y);
                        } else if (EPI == EPI_RESID) {
                            const A2 yy = St<S>::ld(word<S2>(r ? yw.y : yw.x));
                            res = mk2<A2>(yy.x - xx.x + a * v.x, yy.y - xx.y + a * v.y);
                        } else {
                            res = mk2<A2>(xx.x - a * v.x, xx.y - a * v.y);
                        }
                        const S2 rs = St<S>::cv(res);
                        res_bits[r] = bits(rs);
                        if (NV > 0) {
                            const A2 rr = St<S>::ld(rs);
                            if (EPI == EPI_RESID) {
                                red[r][0].x += rr.x * rr.x + rr.y * rr.y;
                            } else if (EPI == EPI_SCHUR_R0) {
                                const A2 q = St<S>::ld(word<S2>(r ? yw.y : yw.x));
                                red[r][0].x += q.x * rr.x + q.y * rr.y;
                                red[r][0].y += q.x * rr.y - q.y * rr.x;
                            } else if (EPI == EPI_SCHUR_TS) {
                                red[r][0].x += rr.x * xx.x + rr.y * xx.y;
                                red[r][0].y += rr.x * xx.y - rr.y * xx.x;
                                red[r][NV - 1].x += rr.x * rr.x + rr.y * rr.y;
                            }
                        }
                    }
                    out2[o] = make_uint2(res_bits[0], res_bits[1]);
                }
            }
    }
    if constexpr (NV > 0) grid_reduce_pairs<NV>(red, MR, p.red);
}

template <int NC, typename S, int MR, bool BLK>
int launch16p_l(const HopParams& p, bool dagger, int epi, cudaStream_t st) {
    if (dagger && epi != EPI_PLAIN && epi != EPI_XPAY)
        return set_error(QCU_ERR_UNSUPPORTED, "dagger hop only with plain/xpay epilogue");
    void (*k)(const HopParams) = nullptr;
    switch (epi) {
        case EPI_PLAIN: k = dagger ? hop16p_kernel<NC, S, true, EPI_PLAIN, MR, BLK> : hop16p_kernel<NC, S, false, EPI_PLAIN, MR, BLK>; break;
        case EPI_XPAY: k = dagger ? hop16p_kernel<NC, S, true, EPI_XPAY, MR, BLK> : hop16p_kernel<NC, S, false, EPI_XPAY, MR, BLK>; break;
        case EPI_SCHUR_R0: k = hop16p_kernel<NC, S, false, EPI_SCHUR_R0, MR, BLK>; break;
        case EPI_SCHUR_TS: k = hop16p_kernel<NC, S, false, EPI_SCHUR_TS, MR, BLK>; break;
        case EPI_SCHUR: k = hop16p_kernel<NC, S, false, EPI_SCHUR, MR, BLK>; break;
        case EPI_RESID: k = hop16p_kernel<NC, S, false, EPI_RESID, MR, BLK>; break;
        default: return set_error(QCU_ERR_INVALID, "epilogue %d", epi);
    }
    constexpr int M2 = MR / 2;
    const int block = (kH16Threads / M2) * M2;
    const int nx = epi == EPI_PLAIN ? 0 : ((epi == EPI_SCHUR_R0 || epi == EPI_RESID) ? 2 : 1);
    const size_t smem = (size_t)nx * kNs * NC * block * sizeof(uint2);   // at most 48 KB
    int grid = resident_grid(k, block, p.g.vh * M2, smem);
    if (grid > kScratchBlocks) grid = kScratchBlocks;
    k<<<grid, block, smem, st>>>(p);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

template <int NC, typename S, int MR>
int launch16p(const HopParams& p, bool dagger, int epi, cudaStream_t st) {
    return p.blocked ? launch16p_l<NC, S, MR, true>(p, dagger, epi, st) : launch16p_l<NC, S, MR, false>(p, dagger, epi, st);
}

// RHS counts with a compile-time specialisation (SU(3) only; other shapes use runtime m)
template <int NC, typename S, bool ACC16>
int launch16d(const HopParams& p, bool dagger, int epi, cudaStream_t st) {
    if constexpr (NC == 3) {
        switch (p.m) {
            case 8: return launch16d_m<NC, S, ACC16, 8>(p, dagger, epi, st);
            case 12: return launch16d_m<NC, S, ACC16, 12>(p, dagger, epi, st);
            case 16: return launch16d_m<NC, S, ACC16, 16>(p, dagger, epi, st);
            default: break;
        }
    }
    return launch16d_m<NC, S, ACC16, 0>(p, dagger, epi, st);
}

template <int NC, typename S, bool ACC16>
int launch16(const HopParams& p, bool dagger, int epi, cudaStream_t st) {
    if (dagger && epi != EPI_PLAIN && epi != EPI_XPAY)
        return set_error(QCU_ERR_UNSUPPORTED, "dagger hop only with plain/xpay epilogue");
    const int spb = std::min(kH16Threads / p.m, kH16MaxSites);
    const int block = spb * p.m;
    void (*k)(const HopParams) = nullptr;
    switch (epi) {
        case EPI_PLAIN: k = dagger ? hop16_kernel<NC, S, true, EPI_PLAIN, ACC16> : hop16_kernel<NC, S, false, EPI_PLAIN, ACC16>; break;
        case EPI_XPAY: k = dagger ? hop16_kernel<NC, S, true, EPI_XPAY, ACC16> : hop16_kernel<NC, S, false, EPI_XPAY, ACC16>; break;
        case EPI_SCHUR_R0: k = hop16_kernel<NC, S, false, EPI_SCHUR_R0, ACC16>; break;
        case EPI_SCHUR_TS: k = hop16_kernel<NC, S, false, EPI_SCHUR_TS, ACC16>; break;
        case EPI_SCHUR: k = hop16_kernel<NC, S, false, EPI_SCHUR, ACC16>; break;
        case EPI_RESID: k = hop16_kernel<NC, S, false, EPI_RESID, ACC16>; break;
        default: return set_error(QCU_ERR_INVALID, "epilogue %d", epi);
    }
    const int64_t want = (p.g.vh + spb - 1) / spb;
    int grid = resident_grid(k, block, p.g.vh * p.m);
    if (grid > want) grid = (int)want;
    if (grid > kScratchBlocks) grid = kScratchBlocks;   // reduction partials: one slot per block
    k<<<grid, block, 0, st>>>(p);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

}  // namespace

bool hop16_supported(int nc, int m, int prec) {
    return (prec == QCU_PRECISION_HALF || prec == QCU_PRECISION_BF16) && nc >= 2 && nc <= 4 && m >= 2 &&
           m <= kH16Threads;
}

// SU(3) shapes with a two-RHS-per-thread specialisation
bool hop16_pairs_supported(int nc, int m, int prec) {
    return (prec == QCU_PRECISION_HALF || prec == QCU_PRECISION_BF16) && nc == 3 && (m == 8 || m == 12 || m == 16);
}

// The epilogues that stage two operands (x and r0) use 47 KB of dynamic shared memory,
// which with the reduction's static arrays is above the 48 KB a kernel gets without
// opting in.  The opt-in is a function attribute; it is set once per process, outside
// any graph capture (context creation, or the first direct launch).
template <typename S, int MR, bool BLK>
static cudaError_t hop16p_optin() {
    constexpr size_t need = (size_t)2 * kNs * 3 * kH16Threads * sizeof(uint2);
    cudaError_t e = cudaFuncSetAttribute(hop16p_kernel<3, S, false, EPI_SCHUR_R0, MR, BLK>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(hop16p_kernel<3, S, false, EPI_RESID, MR, BLK>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need);
    return e;
}

int hop16_pairs_prepare() {
    static bool done = false;
    if (done) return QCU_SUCCESS;
    cudaError_t e = cudaSuccess;
    auto all = [&](auto tag) {
        using S = decltype(tag);
        if (e == cudaSuccess) e = hop16p_optin<S, 8, false>();
        if (e == cudaSuccess) e = hop16p_optin<S, 12, false>();
        if (e == cudaSuccess) e = hop16p_optin<S, 16, false>();
        if (e == cudaSuccess) e = hop16p_optin<S, 8, true>();
        if (e == cudaSuccess) e = hop16p_optin<S, 12, true>();
        if (e == cudaSuccess) e = hop16p_optin<S, 16, true>();
    };
    all(__half{});
    all(__nv_bfloat16{});
    if (e != cudaSuccess) return set_error(QCU_ERR_CUDA, "hop kernel shared-memory opt-in: %s", cudaGetErrorString(e));
    done = true;
    return QCU_SUCCESS;
}

bool hop16_blocked_supported(int nc, int m, int prec, int64_t vh) {
    return hop16_pairs_supported(nc, m, prec) && vh % kSiteBlock == 0 && vh * 4 * nc * m < ((int64_t)1 << 31);
}

int hop16_pairs_launch(const HopParams& p, int nc, int prec, bool dagger, int epi, cudaStream_t st) {
    if (!hop16_pairs_supported(nc, p.m, prec))
        return set_error(QCU_ERR_UNSUPPORTED, "two-RHS packed hop: n_color %d, m %d", nc, p.m);
    if (int rc = hop16_pairs_prepare()) return rc;
    if (p.blocked && !hop16_blocked_supported(nc, p.m, prec, p.g.vh))
        return set_error(QCU_ERR_UNSUPPORTED, "site-blocked layout: half volume %lld", (long long)p.g.vh);
    if (p.g.vh >= (int64_t)1 << 31) return set_error(QCU_ERR_UNSUPPORTED, "half volume beyond 2^31");
    auto go = [&](auto tag) -> int {
        using S = decltype(tag);
        switch (p.m) {
            case 8: return launch16p<3, S, 8>(p, dagger, epi, st);
            case 12: return launch16p<3, S, 12>(p, dagger, epi, st);
            default: return launch16p<3, S, 16>(p, dagger, epi, st);
        }
    };
    if (prec == QCU_PRECISION_HALF) return go(__half{});
    return go(__nv_bfloat16{});
}

// acc16: accumulate the 8 hops in the storage format (FP16 only); staged: read the links
// through the shared-memory staging pass (else every thread reads its own)
int hop16_launch(const HopParams& p, int nc, int prec, bool dagger, int epi, bool acc16, bool staged,
                 cudaStream_t st) {
    if (!hop16_supported(nc, p.m, prec)) return set_error(QCU_ERR_UNSUPPORTED, "packed 16-bit hop: n_color %d, m %d", nc, p.m);
    if (p.g.vh >= (int64_t)1 << 31) return set_error(QCU_ERR_UNSUPPORTED, "half volume beyond 2^31");
    const bool a16 = acc16 && prec == QCU_PRECISION_HALF;
#define QCUB_H16_NC(NCV, SV, A16) (staged ? launch16<NCV, SV, A16>(p, dagger, epi, st) : launch16d<NCV, SV, A16>(p, dagger, epi, st))
    if (prec == QCU_PRECISION_HALF) {
        switch (nc) {
            case 2: return a16 ? QCUB_H16_NC(2, __half, true) : QCUB_H16_NC(2, __half, false);
            case 3: return a16 ? QCUB_H16_NC(3, __half, true) : QCUB_H16_NC(3, __half, false);
            default: return a16 ? QCUB_H16_NC(4, __half, true) : QCUB_H16_NC(4, __half, false);
        }
    }
    switch (nc) {
        case 2: return QCUB_H16_NC(2, __nv_bfloat16, false);
        case 3: return QCUB_H16_NC(3, __nv_bfloat16, false);
        default: return QCUB_H16_NC(4, __nv_bfloat16, false);
    }
#undef QCUB_H16_NC
}

}  // namespace qcub
