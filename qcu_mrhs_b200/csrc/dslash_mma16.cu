// dslash_mma16.cu -- multi-RHS hop term for FP16 / BF16 storage with the link products on
// the warp-level tensor-core MMA (mma.sync m16n8k16, 16-bit operands, FP32 accumulators).
//
// Same operator, layouts and epilogues as dslash_impl.cuh (reference
// include/kernel/su_n_m_rhs_dslash.cuh:92-105, complex_matmul.cuh:16-600; the reference's
// own multi-RHS hop runs its link products through wmma tiles the same way).
//
// One warp per half-site, SU(3), m = 8, 12 or 16 RHS.  For a direction mu the forward and
// the backward hop form one K = 16 contraction (8 complex: forward colours 0..2 + pad,
// backward colours 0..2 + pad), computed as a real 16 x 16 x 8 MMA:
//   rows (M)    RHS: row g <-> RHS 2g, row g + 8 <-> RHS 2g + 1
//   K           (hop, colour, re/im) of the projected half spinor h
//   columns (N) (output colour c', re/im), c' < 3
// B is the real embedding of the hop's matrix W (U forward, U^dag backward):
//   B[(c,re)][(c',re)] = W.re[c'][c]   B[(c,im)][(c',re)] = -W.im[c'][c]
//   B[(c,re)][(c',im)] = W.im[c'][c]   B[(c,im)][(c',im)] =  W.re[c'][c]
// The spin reconstruction needs no arithmetic: spins 0, 1 take the projected half spinors
// h0, h1 as they are, and spins 2, 3 take h0 or h1 times a phase in {+-1, +-i}, which is
// folded into B (c W for c = +-1, +-i).  So each direction is four MMAs, one per output
// spin, all accumulating in FP32 over the 8 hops; the 8 hops cost no SIMT multiply-adds,
// no 16 -> 32-bit conversions and no reconstruction adds.
//
// Fragment layouts (PTX ISA, mma.m16n8k16 with 16-bit A/B): lane = 4 g + t holds
//   A: a0 = (row g, k 2t..2t+1), a1 = (row g+8, k 2t..), a2 = (row g, k 2t+8..), a3 = (row g+8, k 2t+8..)
//   B: b0 = (k 2t..2t+1, col g), b1 = (k 2t+8..2t+9, col g)
//   D: d0, d1 = (row g, col 2t..2t+1), d2, d3 = (row g+8, col 2t..2t+1)
// so lane (g, t) loads the neighbour spinor words of colour t for RHS 2g and 2g+1 (one
// 8-byte load per spin: the two RHS are adjacent in the gathered layout), the link element
// W[g/2][t], and ends with the output of colour t for RHS 2g and 2g+1 in FP32.  Lanes with
// t = 3 (colour pad), g >= 6 (column pad) or 2g >= m hold zeros where they would load.
#include "dslash.h"
#include "dslash_impl.cuh"
#include "workspace.h"

namespace qcub {

namespace {

constexpr int kMmaThreads = 256;
constexpr int kMmaWarps = kMmaThreads / 32;

template <typename S> struct M16;
template <> struct M16<__half> {
    using T2 = __half2;
    __device__ static void mma(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                               uint32_t b1) {
        asm("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
    }
    __device__ static uint32_t add(uint32_t a, uint32_t b) {
        __half2 r = __hadd2(*reinterpret_cast<__half2*>(&a), *reinterpret_cast<__half2*>(&b));
        return *reinterpret_cast<uint32_t*>(&r);
    }
    __device__ static uint32_t sub(uint32_t a, uint32_t b) {
        __half2 r = __hsub2(*reinterpret_cast<__half2*>(&a), *reinterpret_cast<__half2*>(&b));
        return *reinterpret_cast<uint32_t*>(&r);
    }
};
template <> struct M16<__nv_bfloat16> {
    using T2 = __nv_bfloat162;
    __device__ static void mma(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                               uint32_t b1) {
        asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
    }
    __device__ static uint32_t add(uint32_t a, uint32_t b) {
        __nv_bfloat162 r = __hadd2(*reinterpret_cast<__nv_bfloat162*>(&a), *reinterpret_cast<__nv_bfloat162*>(&b));
        return *reinterpret_cast<uint32_t*>(&r);
    }
    __device__ static uint32_t sub(uint32_t a, uint32_t b) {
        __nv_bfloat162 r = __hsub2(*reinterpret_cast<__nv_bfloat162*>(&a), *reinterpret_cast<__nv_bfloat162*>(&b));
        return *reinterpret_cast<uint32_t*>(&r);
    }
};

// packed complex words: re in the low half, im in the high half
__device__ __forceinline__ uint32_t mi_times_i(uint32_t u) { return __byte_perm(u, 0, 0x1032) ^ 0x00008000u; }   // i v
__device__ __forceinline__ uint32_t mi_times_mi(uint32_t u) { return __byte_perm(u, 0, 0x1032) ^ 0x80000000u; }  // -i v
__device__ __forceinline__ uint32_t neg2(uint32_t u) { return u ^ 0x80008000u; }

// Spin projection of one RHS's neighbour words p0..p3 (same colour) for direction MU with
// projector 1 - SG g_MU (DeGrand-Rossi basis, the tables of dslash_impl.cuh).
template <typename S, int MU, int SG>
__device__ __forceinline__ void mma_project(uint32_t p0, uint32_t p1, uint32_t p2, uint32_t p3, uint32_t& h0,
                                            uint32_t& h1) {
    using P = M16<S>;
    if (MU == 0) {        // h0 = p0 + s i p3 ; h1 = p1 + s i p2
        h0 = P::add(p0, SG > 0 ? mi_times_i(p3) : mi_times_mi(p3));
        h1 = P::add(p1, SG > 0 ? mi_times_i(p2) : mi_times_mi(p2));
    } else if (MU == 1) { // h0 = p0 - s p3 ; h1 = p1 + s p2
        h0 = SG > 0 ? P::sub(p0, p3) : P::add(p0, p3);
        h1 = SG > 0 ? P::add(p1, p2) : P::sub(p1, p2);
    } else if (MU == 2) { // h0 = p0 + s i p2 ; h1 = p1 - s i p3
        h0 = P::add(p0, SG > 0 ? mi_times_i(p2) : mi_times_mi(p2));
        h1 = P::add(p1, SG > 0 ? mi_times_mi(p3) : mi_times_i(p3));
    } else {              // h0 = p0 + s p2 ; h1 = p1 + s p3
        h0 = SG > 0 ? P::add(p0, p2) : P::sub(p0, p2);
        h1 = SG > 0 ? P::add(p1, p3) : P::sub(p1, p3);
    }
}

// Lane constants of the B embedding: column part (re or im of c') decides which half of
// the link word goes where.  emb(W) and emb(i W) as one byte permute and one sign mask.
struct EmbLane {
    uint32_t sel_w, msk_w;   // emb(W)   = perm(W, sel_w) ^ msk_w
    uint32_t sel_i, msk_i;   // emb(i W) = perm(W, sel_i) ^ msk_i
};
__device__ __forceinline__ EmbLane emb_lane(int part) {
    // part re: emb(W) = (W.re, -W.im), emb(iW) = (-W.im, -W.re)
    // part im: emb(W) = (W.im,  W.re), emb(iW) = ( W.re, -W.im)
    EmbLane e;
    e.sel_w = part ? 0x1032u : 0x3210u;
    e.msk_w = part ? 0u : 0x80000000u;
    e.sel_i = part ? 0x3210u : 0x1032u;
    e.msk_i = part ? 0x80000000u : 0x80008000u;
    return e;
}
// emb(c W) for the phase code C: 0 = +1, 1 = -1, 2 = +i, 3 = -i
template <int C>
__device__ __forceinline__ uint32_t emb(uint32_t w, const EmbLane& e) {
    if (C == 0) return __byte_perm(w, 0, e.sel_w) ^ e.msk_w;
    if (C == 1) return __byte_perm(w, 0, e.sel_w) ^ e.msk_w ^ 0x80008000u;
    if (C == 2) return __byte_perm(w, 0, e.sel_i) ^ e.msk_i;
    return __byte_perm(w, 0, e.sel_i) ^ e.msk_i ^ 0x80008000u;
}
// phase code of -c
__host__ __device__ constexpr int neg_code(int c) { return c ^ 1; }
// phase code of s (s = +-1) times the unit u (u = 1 or i): s*1 -> 0/1, s*i -> 2/3
__host__ __device__ constexpr int phase(int s, bool imag) { return (imag ? 2 : 0) + (s > 0 ? 0 : 1); }

// Lower-spin phases of the reconstruction for direction MU and projector sign SG
// (spin 2 += C2 w_{P2}, spin 3 += C3 w_{P3}, w_k = W h_k):
//   MU 0: spin2 += -s i w1, spin3 += -s i w0      MU 1: spin2 += s w1, spin3 += -s w0
//   MU 2: spin2 += -s i w0, spin3 +=  s i w1      MU 3: spin2 += s w0, spin3 +=  s w1
template <int MU, int SG> struct Recon {
    static constexpr int P2 = MU <= 1 ? 1 : 0;
    static constexpr int P3 = 1 - P2;
    static constexpr int C2 = MU == 0 ? phase(-SG, true) : MU == 1 ? phase(SG, false)
                            : MU == 2 ? phase(-SG, true) : phase(SG, false);
    static constexpr int C3 = MU == 0 ? phase(-SG, true) : MU == 1 ? phase(-SG, false)
                            : MU == 2 ? phase(SG, true) : phase(SG, false);
};

// One direction: forward neighbour words qf[s] (RHS 2g in .x, 2g+1 in .y), backward qb[s],
// link words wf = W_f[g/2][t], wb = W_b[g/2][t].
template <typename S, int MU, int SF>
__device__ __forceinline__ void mma_dir(float (&d)[4][4], const uint2 (&qf)[4], const uint2 (&qb)[4], uint32_t wf,
                                        uint32_t wb, const EmbLane& e) {
    constexpr int SB = -SF;
    using P = M16<S>;
    uint32_t hf[2][2], hb[2][2];   // [k][rhs of the pair]
    mma_project<S, MU, SF>(qf[0].x, qf[1].x, qf[2].x, qf[3].x, hf[0][0], hf[1][0]);
    mma_project<S, MU, SF>(qf[0].y, qf[1].y, qf[2].y, qf[3].y, hf[0][1], hf[1][1]);
    mma_project<S, MU, SB>(qb[0].x, qb[1].x, qb[2].x, qb[3].x, hb[0][0], hb[1][0]);
    mma_project<S, MU, SB>(qb[0].y, qb[1].y, qb[2].y, qb[3].y, hb[0][1], hb[1][1]);
    using RF = Recon<MU, SF>;
    using RB = Recon<MU, SB>;
    const uint32_t bf = emb<0>(wf, e), bb = emb<0>(wb, e);
    P::mma(d[0], hf[0][0], hf[0][1], hb[0][0], hb[0][1], bf, bb);
    P::mma(d[1], hf[1][0], hf[1][1], hb[1][0], hb[1][1], bf, bb);
    const uint32_t b2f = emb<RF::C2>(wf, e), b2b = emb<RB::C2>(wb, e);
    P::mma(d[2], hf[RF::P2][0], hf[RF::P2][1], hb[RB::P2][0], hb[RB::P2][1], b2f, b2b);
    uint32_t b3f, b3b;
    if (RF::C3 == RF::C2) { b3f = b2f; b3b = b2b; }
    else if (RF::C3 == neg_code(RF::C2)) { b3f = neg2(b2f); b3b = neg2(b2b); }
    else { b3f = emb<RF::C3>(wf, e); b3b = emb<RB::C3>(wb, e); }
    P::mma(d[3], hf[RF::P3][0], hf[RF::P3][1], hb[RB::P3][0], hb[RB::P3][1], b3f, b3b);
}

template <typename S, bool DAG, int EPI, int MR>
__global__ void __launch_bounds__(kMmaThreads, 2) hop_mma16_kernel(const HopParams p) {
    constexpr int NC = 3;
    constexpr int N2 = NC * NC;
    constexpr int NV = (EPI == EPI_SCHUR_R0 || EPI == EPI_RESID) ? 1 : (EPI == EPI_SCHUR_TS ? 2 : 0);
    constexpr int SF = DAG ? 1 : -1;   // forward projector 1 - s g: sign of gamma
    constexpr int SB = DAG ? -1 : 1;
    constexpr int SITE = 4 * NC * MR;  // 32-bit words of one site
    static_assert(MR % 2 == 0 && MR <= 16, "one warp covers up to 16 RHS in pairs");
    using S2 = typename St<S>::S2;
    if (skip_launch(p.done, p.gate)) return;
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const bool ld_ok = t < NC && 2 * g < MR;          // this lane's spinor words exist
    const bool w_ok = t < NC && g < 2 * NC;           // this lane's link element exists
    const int woff = (g >> 1) * NC + t;               // forward: U[g/2][t]
    const int woff_b = t * NC + (g >> 1);             // backward: U[t][g/2], conjugated
    const EmbLane e = emb_lane(g & 1);
    const int64_t vh = p.g.vh;
    const int parity = p.parity;
    const uint32_t* __restrict__ in = static_cast<const uint32_t*>(p.in);
    const uint32_t* __restrict__ gauge = static_cast<const uint32_t*>(p.gauge);
    const uint32_t* gf = gauge + (int64_t)parity * vh * N2;
    const uint32_t* gb = gauge + (int64_t)(1 - parity) * vh * N2;
    const int64_t gmu = 2 * vh * N2;
    const uint32_t tflip = p.t_sign < 0 ? 0x80008000u : 0u;
    const int lxh = p.g.lxh, Ly = p.g.L[1], Lz = p.g.L[2], Lt = p.g.L[3];
    const int64_t sy = lxh, sz = (int64_t)lxh * Ly, st = sz * Lz;
    const int lofs = t * MR + 2 * g;                  // word offset of (spin 0, colour t, RHS 2g)
    float2 red[2][NV > 0 ? NV : 1];
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int k = 0; k < (NV > 0 ? NV : 1); ++k) red[q][k] = make_float2(0.f, 0.f);

    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    // neighbour half-site indices of a site (forward, backward per direction) and whether
    // its t hops cross the boundary
    auto neighbours = [&](int64_t site, uint32_t (&nb)[8], bool& wf_t, bool& wb_t) {
        const SiteXYZT c = site_coords(p.g, (uint32_t)site);
        const int xodd = (parity ^ (c.y + c.z + c.t)) & 1;
        nb[0] = (uint32_t)(site - c.xh + (xodd ? (c.xh + 1 == lxh ? 0 : c.xh + 1) : c.xh));
        nb[1] = (uint32_t)(site - c.xh + (xodd ? c.xh : (c.xh == 0 ? lxh - 1 : c.xh - 1)));
        nb[2] = (uint32_t)(site + (c.y + 1 == Ly ? -(int64_t)(Ly - 1) * sy : sy));
        nb[3] = (uint32_t)(site + (c.y == 0 ? (int64_t)(Ly - 1) * sy : -sy));
        nb[4] = (uint32_t)(site + (c.z + 1 == Lz ? -(int64_t)(Lz - 1) * sz : sz));
        nb[5] = (uint32_t)(site + (c.z == 0 ? (int64_t)(Lz - 1) * sz : -sz));
        wf_t = (c.t + 1 == Lt);
        wb_t = (c.t == 0);
        nb[6] = (uint32_t)(site + (wf_t ? -(int64_t)(Lt - 1) * st : st));
        nb[7] = (uint32_t)(site + (wb_t ? (int64_t)(Lt - 1) * st : -st));
    };
    for (int64_t site = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; site < vh; site += nwarps) {
        uint32_t nbr[8];
        bool wf_t, wb_t;
        neighbours(site, nbr, wf_t, wb_t);
        float d[4][4];
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
            for (int k = 0; k < 4; ++k) d[s][k] = 0.f;

        auto load_dir = [&](int mu, uint2 (&qf)[4], uint2 (&qb)[4], uint32_t& wf, uint32_t& wb) {
            const uint2* pf = reinterpret_cast<const uint2*>(in + (int64_t)nbr[2 * mu] * SITE + lofs);
            const uint2* pb = reinterpret_cast<const uint2*>(in + (int64_t)nbr[2 * mu + 1] * SITE + lofs);
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                qf[s] = ld_ok ? __ldg(pf + s * (NC * MR / 2)) : make_uint2(0u, 0u);
                qb[s] = ld_ok ? __ldg(pb + s * (NC * MR / 2)) : make_uint2(0u, 0u);
            }
            const uint32_t ff = (mu == 3 && wf_t) ? tflip : 0u;
            const uint32_t fb = (mu == 3 && wb_t) ? tflip : 0u;
            wf = w_ok ? (__ldg(gf + mu * gmu + site * N2 + woff) ^ ff) : 0u;
            wb = w_ok ? (__ldg(gb + mu * gmu + (int64_t)nbr[2 * mu + 1] * N2 + woff_b) ^ 0x80000000u ^ fb) : 0u;
        };
        // all 8 neighbours' words and links are requested before the first MMA, so a site
        // costs one memory round trip instead of four
        uint2 qf[4][4], qb[4][4];
        uint32_t wf[4], wb[4];
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) load_dir(mu, qf[mu], qb[mu], wf[mu], wb[mu]);
        mma_dir<S, 0, SF>(d, qf[0], qb[0], wf[0], wb[0], e);
        mma_dir<S, 1, SF>(d, qf[1], qb[1], wf[1], wb[1], e);
        mma_dir<S, 2, SF>(d, qf[2], qb[2], wf[2], wb[2], e);
        mma_dir<S, 3, SF>(d, qf[3], qb[3], wf[3], wb[3], e);
        (void)SB;

        // epilogue: lane (g, t) owns colour t of RHS 2g (d[s][0..1]) and 2g+1 (d[s][2..3])
        if (ld_ok) {
            uint2* __restrict__ out2 = reinterpret_cast<uint2*>(static_cast<uint32_t*>(p.out) + site * SITE + lofs);
            const uint2* x2 = reinterpret_cast<const uint2*>(static_cast<const uint32_t*>(p.x) + site * SITE + lofs);
            const uint2* y2 = reinterpret_cast<const uint2*>(static_cast<const uint32_t*>(p.r0) + site * SITE + lofs);
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const float2 v0 = make_float2(d[s][0], d[s][1]), v1 = make_float2(d[s][2], d[s][3]);
                if (EPI == EPI_PLAIN) {
                    const S2 o0 = St<S>::cv(v0), o1 = St<S>::cv(v1);
                    out2[s * (NC * MR / 2)] = make_uint2(*reinterpret_cast<const uint32_t*>(&o0),
                                                         *reinterpret_cast<const uint32_t*>(&o1));
                } else {
                    const uint2 xw = __ldg(x2 + s * (NC * MR / 2));
                    uint2 yw = make_uint2(0u, 0u);
                    if (EPI == EPI_RESID || EPI == EPI_SCHUR_R0) yw = __ldg(y2 + s * (NC * MR / 2));
                    uint32_t res_bits[2];
#pragma unroll
                    for (int r = 0; r < 2; ++r) {
                        const float2 v = r ? v1 : v0;
                        const uint32_t xb = r ? xw.y : xw.x, yb = r ? yw.y : yw.x;
                        const float2 xx = St<S>::ld(*reinterpret_cast<const S2*>(&xb));
                        const float a = (float)p.a;
                        float2 res;
                        if (EPI == EPI_XPAY) {
                            res = make_float2(xx.x + a * v.x, xx.y + a * v.y);
                        } else if (EPI == EPI_RESID) {
                            const float2 yy = St<S>::ld(*reinterpret_cast<const S2*>(&yb));
                            res = make_float2(yy.x - xx.x + a * v.x, yy.y - xx.y + a * v.y);
                        } else {
                            res = make_float2(xx.x - a * v.x, xx.y - a * v.y);
                        }
                        const S2 rs = St<S>::cv(res);
                        res_bits[r] = *reinterpret_cast<const uint32_t*>(&rs);
                        if (NV > 0) {
                            const float2 rr = St<S>::ld(rs);
                            if (EPI == EPI_RESID) {
                                red[r][0].x += rr.x * rr.x + rr.y * rr.y;
                            } else if (EPI == EPI_SCHUR_R0) {   // <r0, out> = sum conj(r0) out
                                const float2 q = St<S>::ld(*reinterpret_cast<const S2*>(&yb));
                                red[r][0].x += q.x * rr.x + q.y * rr.y;
                                red[r][0].y += q.x * rr.y - q.y * rr.x;
                            } else if (EPI == EPI_SCHUR_TS) {  // <out, x>, <out, out>
                                red[r][0].x += rr.x * xx.x + rr.y * xx.y;
                                red[r][0].y += rr.x * xx.y - rr.y * xx.x;
                                red[r][NV - 1].x += rr.x * rr.x + rr.y * rr.y;
                            }
                        }
                    }
                    out2[s * (NC * MR / 2)] = make_uint2(res_bits[0], res_bits[1]);
                }
            }
        }
    }
    if constexpr (NV > 0) {
        // lanes 4g..4g+3 hold RHS 2g, 2g+1: sum over t (fixed order), then over the block's
        // warps in order, then the common grid stage
        __shared__ double2 wsum[kMmaWarps][NV][16];
        __shared__ double2 bsum[NV * kMaxRhs];
        const int warp = threadIdx.x >> 5;
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                double vx = (double)red[r][k].x, vy = (double)red[r][k].y;
                vx += __shfl_xor_sync(0xffffffffu, vx, 1);
                vy += __shfl_xor_sync(0xffffffffu, vy, 1);
                vx += __shfl_xor_sync(0xffffffffu, vx, 2);
                vy += __shfl_xor_sync(0xffffffffu, vy, 2);
                if (t == 0 && 2 * g < MR) wsum[warp][k][2 * g + r] = make_double2(vx, vy);
            }
        __syncthreads();
        for (int idx = threadIdx.x; idx < NV * MR; idx += blockDim.x) {
            const int k = idx / MR, rhs = idx - k * MR;
            double2 s = make_double2(0.0, 0.0);
            for (int w = 0; w < kMmaWarps; ++w) {
                s.x += wsum[w][k][rhs].x;
                s.y += wsum[w][k][rhs].y;
            }
            bsum[idx] = s;
        }
        __syncthreads();
        publish_and_finish<NV>(bsum, MR, p.red);
    }
}

template <typename S, int MR>
int launch_mma16(const HopParams& p, bool dagger, int epi, cudaStream_t st) {
    if (dagger && epi != EPI_PLAIN && epi != EPI_XPAY)
        return set_error(QCU_ERR_UNSUPPORTED, "dagger hop only with plain/xpay epilogue");
    void (*k)(const HopParams) = nullptr;
    switch (epi) {
        case EPI_PLAIN: k = dagger ? hop_mma16_kernel<S, true, EPI_PLAIN, MR> : hop_mma16_kernel<S, false, EPI_PLAIN, MR>; break;
        case EPI_XPAY: k = dagger ? hop_mma16_kernel<S, true, EPI_XPAY, MR> : hop_mma16_kernel<S, false, EPI_XPAY, MR>; break;
        case EPI_SCHUR_R0: k = hop_mma16_kernel<S, false, EPI_SCHUR_R0, MR>; break;
        case EPI_SCHUR_TS: k = hop_mma16_kernel<S, false, EPI_SCHUR_TS, MR>; break;
        case EPI_SCHUR: k = hop_mma16_kernel<S, false, EPI_SCHUR, MR>; break;
        case EPI_RESID: k = hop_mma16_kernel<S, false, EPI_RESID, MR>; break;
        default: return set_error(QCU_ERR_INVALID, "epilogue %d", epi);
    }
    int grid = resident_grid(k, kMmaThreads, p.g.vh * 32);
    if (grid > kScratchBlocks) grid = kScratchBlocks;
    k<<<grid, kMmaThreads, 0, st>>>(p);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

template <typename S>
int launch_mma16_m(const HopParams& p, bool dagger, int epi, cudaStream_t st) {
    switch (p.m) {
        case 8: return launch_mma16<S, 8>(p, dagger, epi, st);
        case 12: return launch_mma16<S, 12>(p, dagger, epi, st);
        case 16: return launch_mma16<S, 16>(p, dagger, epi, st);
        default: return set_error(QCU_ERR_UNSUPPORTED, "tensor-core 16-bit hop: m_rhs=%d (8, 12, 16)", p.m);
    }
}

}  // namespace

bool hop_mma16_supported(int nc, int m, int prec) {
    return nc == 3 && (m == 8 || m == 12 || m == 16) &&
           (prec == QCU_PRECISION_HALF || prec == QCU_PRECISION_BF16);
}

int hop_mma16_launch(const HopParams& p, int nc, int prec, bool dagger, int epi, cudaStream_t st) {
    if (!hop_mma16_supported(nc, p.m, prec))
        return set_error(QCU_ERR_UNSUPPORTED, "tensor-core 16-bit hop: n_color=%d m_rhs=%d precision=%d", nc, p.m,
                         prec);
    if (reinterpret_cast<uintptr_t>(p.in) % 8 || reinterpret_cast<uintptr_t>(p.out) % 8 ||
        (p.x && reinterpret_cast<uintptr_t>(p.x) % 8) || (p.r0 && reinterpret_cast<uintptr_t>(p.r0) % 8))
        return set_error(QCU_ERR_INVALID, "tensor-core 16-bit hop: vectors must be 8-byte aligned");
    if (prec == QCU_PRECISION_HALF) return launch_mma16_m<__half>(p, dagger, epi, st);
    return launch_mma16_m<__nv_bfloat16>(p, dagger, epi, st);
}

}  // namespace qcub
