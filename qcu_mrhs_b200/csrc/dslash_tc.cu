// dslash_tc.cu -- multi-RHS hop term on the 5th-generation tensor cores (tcgen05),
// for FP16 and BF16 storage with FP32 accumulation in tensor memory.
//
// Same operator and layouts as dslash_impl.cuh (reference
// include/kernel/su_n_m_rhs_dslash.cuh:92-105, complex_matmul.cuh:16-600).
//
// Formulation.  For a site x and one of its 8 hops h, the contribution to out(x) is
//   out_h[s][c][r] = sum_c' W_h[c][c'] * P_h[s][c'][r],   P_h = (1 -+ s g_mu) psi(x +- mu)
// (W_h = U_mu(x) forward, U_mu(x-mu)^dagger backward).  The 4-spinor projection P_h is
// formed row by row; (s, r) rows share the link, so this is a real GEMM with
//   M = rows (site, s, r),  K = (c', re/im),  N = (c, re/im)
// and B = the real embedding of W_h^T.  Two sites share one M = 128 tile when
// 4m <= 64 and 2N <= 8: their K and N ranges are disjoint blocks (B block-diagonal),
// so one instruction computes both sites' hop.  All 8 hops accumulate into the same
// tensor-memory tile.
//
// Data path per tile (one CTA = 128 threads = 128 tile rows, thread i <-> TMEM lane i):
//   A  (128 x 16 bf16/f16) in TMEM: each thread projects its row in packed 16-bit
//      arithmetic and writes it with tcgen05.st (8 x 32-bit columns);
//   B  (16 x 16) in shared memory, K-major, no swizzle: written from the links;
//   D  (128 x 16 fp32) in TMEM, tcgen05.mma kind::f16 issued by one thread, completion
//      signalled through tcgen05.commit to an mbarrier;
//   per tile: every thread issues the loads of all 8 hops first (they overlap the
//      previous tile's MMAs), then waits for those MMAs, runs the previous tile's
//      epilogue, writes the 8 A rows and 8 B tiles, one barrier, and one thread issues
//      the 8 MMAs back to back and one commit;
//   epilogue: tcgen05.ld of the thread's row, conversion, store (and the fused
//      Schur/xpay epilogues and per-RHS reductions of the SIMT kernel).
// Every wait on an mbarrier is bounded; on timeout the kernel records an error code
// and finishes (results are then invalid, never a hang).
#include "dslash.h"
#include "dslash_impl.cuh"
#include "workspace.h"

namespace qcub {

int* device_error_flag();   // runtime.cu: per-device flag, nonzero after a timed-out wait

namespace tc {

constexpr int kThreads = 128;
constexpr int kTmemCols = 128;         // D: 16 columns, A: 8 hops x 8 columns (80 used)
constexpr int kColD = 0, kColA = 16;
constexpr uint32_t kWaitLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Bounded wait for the phase with the given parity to complete.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t addr = smem_u32(bar);
    for (uint32_t it = 0; it < kWaitLimit; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(addr), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&v)[8]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
        : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// K-major, no-swizzle shared-memory matrix descriptor: 8-row x 16-byte core matrices,
// LBO = byte distance between the two K-adjacent core matrices, SBO = between 8-row groups.
__device__ __forceinline__ uint64_t smem_desc(const void* base, uint32_t lbo, uint32_t sbo) {
    const uint64_t addr = smem_u32(base);
    return ((addr >> 4) & 0x3FFFull) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::f16, D = F32, A/B = F16 (fmt 0) or BF16 (fmt 1), both
// K-major, M = 128, N = 16.
__host__ __device__ constexpr uint32_t instr_desc(uint32_t fmt) {
    return (1u << 4) | (fmt << 7) | (fmt << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
        "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

template <typename S> struct Pk;
template <> struct Pk<__half> {
    using T2 = __half2;
    static constexpr uint32_t fmt = 0;
    __device__ static T2 sgn(float a, float b) { return __floats2half2_rn(a, b); }
};
template <> struct Pk<__nv_bfloat16> {
    using T2 = __nv_bfloat162;
    static constexpr uint32_t fmt = 1;
    __device__ static T2 sgn(float a, float b) { return __floats2bfloat162_rn(a, b); }
};

template <typename T2>
__device__ __forceinline__ uint32_t as_u32(T2 v) {
    return *reinterpret_cast<uint32_t*>(&v);
}
template <typename T2>
__device__ __forceinline__ T2 from_u32(uint32_t u) {
    return *reinterpret_cast<T2*>(&u);
}
__device__ __forceinline__ uint32_t swap_halves(uint32_t u) { return __byte_perm(u, 0, 0x1032); }

// Partner spin p(s) and sign of gamma_mu[s][p(s)] (DeGrand-Rossi, reference qcu_gamma.cuh);
// gamma_1 and gamma_3 entries are imaginary.
__device__ __forceinline__ int partner(int mu, int s) { return mu < 2 ? 3 - s : (s ^ 2); }
__device__ __forceinline__ float gsign(int mu, int s) {
    // mu=0: +i,+i,-i,-i ; mu=1: -1,+1,+1,-1 ; mu=2: +i,-i,-i,+i ; mu=3: +1,+1,+1,+1
    // nibble mu of 0x069C has bit s set where the entry is negative
    return ((0x069Cu >> (4 * mu + s)) & 1u) ? -1.f : 1.f;
}

struct Tile {
    int lxh, Ly, Lz, Lt;
    int64_t vh;
};

// neighbour half-site index of `site` (parity `parity`) in direction mu, forward/backward;
// *wrap is set when the hop crosses the t boundary.
__device__ __forceinline__ int64_t neighbour(const Tile& g, int64_t site, int xh, int y, int z, int t,
                                             int xodd, int mu, bool fwd, bool* wrap) {
    const int64_t sy = g.lxh, sz = (int64_t)g.lxh * g.Ly, st = sz * g.Lz;
    *wrap = false;
    switch (mu) {
        case 0:
            if (fwd) return site - xh + (xodd ? (xh + 1 == g.lxh ? 0 : xh + 1) : xh);
            return site - xh + (xodd ? xh : (xh == 0 ? g.lxh - 1 : xh - 1));
        case 1:
            if (fwd) return site + (y + 1 == g.Ly ? -(int64_t)(g.Ly - 1) * sy : sy);
            return site + (y == 0 ? (int64_t)(g.Ly - 1) * sy : -sy);
        case 2:
            if (fwd) return site + (z + 1 == g.Lz ? -(int64_t)(g.Lz - 1) * sz : sz);
            return site + (z == 0 ? (int64_t)(g.Lz - 1) * sz : -sz);
        default:
            if (fwd) {
                *wrap = (t + 1 == g.Lt);
                return site + (*wrap ? -(int64_t)(g.Lt - 1) * st : st);
            }
            *wrap = (t == 0);
            return site + (*wrap ? (int64_t)(g.Lt - 1) * st : -st);
    }
}

struct SiteCoord {
    int xh, y, z, t, xodd;
};

__device__ __forceinline__ SiteCoord coords(const Geom& geo, int64_t site, int parity) {
    const SiteXYZT q = site_coords(geo, (uint32_t)site);
    SiteCoord c;
    c.xh = q.xh;
    c.y = q.y;
    c.z = q.z;
    c.t = q.t;
    c.xodd = (parity ^ (c.y + c.z + c.t)) & 1;
    return c;
}

// B tile: 16 (n) x 16 (k) 16-bit values, K-major core matrices: (n/8, k/8) at
// (n/8)*256 + (k/8)*128 bytes, row n%8 at +16*(n%8), element k%8 at +2*(k%8).
__device__ __forceinline__ int b_word(int n, int k) {   // 32-bit word index of (n, k..k+1), k even
    return ((n >> 3) * 256 + (k >> 3) * 128 + (n & 7) * 16 + (k & 7) * 2) >> 2;
}

// Projected row value of one hop: row_s = psi_s + coef * psi_p(s) in packed 16-bit math.
template <typename P2>
__device__ __forceinline__ uint32_t project(uint32_t a, uint32_t b, bool imag, P2 cvec) {
    if (imag) b = swap_halves(b);
    return as_u32(__hfma2(from_u32<P2>(b), cvec, from_u32<P2>(a)));
}

template <int NC, typename S, bool DAG, int EPI>
__global__ void __launch_bounds__(kThreads, NC <= 4 ? 4 : 2) hop_tc_kernel(const HopParams p, int* err) {
    using S2 = typename St<S>::S2;
    using A2 = typename St<S>::A2;
    using P2 = typename Pk<S>::T2;
    constexpr int NV = (EPI == EPI_SCHUR_R0 || EPI == EPI_RESID) ? 1 : (EPI == EPI_SCHUR_TS ? 2 : 0);
    constexpr int HG = NC <= 4 ? 8 : 4;   // hops whose operands are held in registers at once
    __shared__ __align__(128) uint32_t sB[8][128];   // one 512-byte B tile per hop
    __shared__ __align__(8) uint64_t sBar;
    __shared__ uint32_t sTmem;
    __shared__ double2 sRed[NV > 0 ? NV * kMaxRhs : 1];
    __shared__ double2 sRow[NV > 0 ? NV * kThreads : 1];

    if (skip_launch(p.done, p.gate)) return;
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int m = p.m;
    const int rows_site = 4 * m;                                   // <= 128
    const int spt = (rows_site <= 64 && 2 * NC <= 8) ? 2 : 1;      // sites per tile
    const int kb = spt == 2 ? 8 : 16;                              // K (and N) block per site
    const Tile g{p.g.lxh, p.g.L[1], p.g.L[2], p.g.L[3], p.g.vh};
    const int64_t ntiles = (g.vh + spt - 1) / spt;
    const int parity = p.parity;
    const S2* __restrict__ in = static_cast<const S2*>(p.in);
    const S2* __restrict__ gauge = static_cast<const S2*>(p.gauge);
    const int64_t site_len = (int64_t)kNs * NC * m;
    constexpr int N2 = NC * NC;
    const int64_t gmu = 2 * g.vh * N2;

    // this thread's tile row (site in tile, spin, RHS)
    const int sl = tid / rows_site;
    const int within = tid - sl * rows_site;
    const int sp = within / m;
    const int rr = within - sp * m;
    const bool row_used = sl < spt;
    const int col0 = sl * (kb >> 1);   // first A column (32-bit) of this row's site block

    // B work item of this thread: (site block, c_out, ri_out, c_in)
    const int nbitems = spt * NC * 2 * NC;
    const bool b_worker = tid < nbitems;
    int b_sl = 0, b_cout = 0, b_riout = 0, b_cin = 0;
    if (b_worker) {
        int q = tid;
        b_cin = q % NC; q /= NC;
        b_riout = q % 2; q /= 2;
        b_cout = q % NC;
        b_sl = q / NC;
    }

    // one-time set-up: barrier, zeroed B tiles, TMEM allocation (D: 16 cols, A: 8 x 8 cols)
    if (tid == 0) {
        mbar_init(&sBar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < 8 * 128; i += kThreads) (&sB[0][0])[i] = 0u;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sTmem)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = sTmem;
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    const uint32_t idesc = instr_desc(Pk<S>::fmt);
    bool timed_out = false;

    double2 red[NV > 0 ? NV : 1];
#pragma unroll
    for (int k = 0; k < (NV > 0 ? NV : 1); ++k) red[k] = make_double2(0.0, 0.0);

    // epilogue of a finished tile: read this thread's D row, write (and reduce) its values
    auto epilogue = [&](int64_t site, bool valid) {
        float d[16];
        tmem_ld16(tmem + lane_base + kColD, d);
        fence_before_sync();
        if (!valid) return;
        S2* __restrict__ out = static_cast<S2*>(p.out);
        const S2* __restrict__ xv = static_cast<const S2*>(p.x);
        const S2* __restrict__ r0v = static_cast<const S2*>(p.r0);
        const int64_t base = site * site_len + rr;
        const int off = sl * kb;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const int64_t o = base + (int64_t)(sp * NC + c) * m;
            float vre = d[2 * c], vim = d[2 * c + 1];
            if (NC <= 4 && off != 0) {
                vre = d[8 + 2 * c];
                vim = d[8 + 2 * c + 1];
            }
            const A2 v = mk2<A2>(vre, vim);
            if (EPI == EPI_PLAIN) {
                out[o] = St<S>::cv(v);
            } else {
                const A2 xx = St<S>::ld(xv[o]);
                const float a = (float)p.a;
                A2 res;
                if (EPI == EPI_XPAY) {
                    res = mk2<A2>(xx.x + a * v.x, xx.y + a * v.y);
                } else if (EPI == EPI_RESID) {
                    const A2 yy = St<S>::ld(r0v[o]);
                    res = mk2<A2>(yy.x - xx.x + a * v.x, yy.y - xx.y + a * v.y);
                } else {
                    res = mk2<A2>(xx.x - a * v.x, xx.y - a * v.y);
                }
                const S2 rs = St<S>::cv(res);
                out[o] = rs;
                if (NV > 0) {
                    const A2 q = St<S>::ld(rs);
                    if (EPI == EPI_RESID) {
                        red[0].x += (double)q.x * q.x + (double)q.y * q.y;
                    } else if (EPI == EPI_SCHUR_R0) {
                        const A2 z = St<S>::ld(r0v[o]);
                        red[0].x += (double)z.x * q.x + (double)z.y * q.y;
                        red[0].y += (double)z.x * q.y - (double)z.y * q.x;
                    } else if (EPI == EPI_SCHUR_TS) {
                        red[0].x += (double)q.x * xx.x + (double)q.y * xx.y;
                        red[0].y += (double)q.x * xx.y - (double)q.y * xx.x;
                        red[NV - 1].x += (double)q.x * q.x + (double)q.y * q.y;
                    }
                }
            }
        }
    };

    // projector 1 + sigma gamma_mu: sigma = -s forward, +s backward (s = -1 with dagger)
    const float sdag = DAG ? -1.f : 1.f;
    uint32_t phase = 0;
    bool pending = false;
    int64_t prev_site = 0;
    bool prev_valid = false;

    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t site0 = tile * spt;
        const int64_t my_site = site0 + sl;
        const bool row_valid = row_used && my_site < g.vh;
        SiteCoord mc{};
        if (row_valid) mc = coords(p.g, my_site, parity);
        const int64_t b_site = site0 + b_sl;
        const bool b_valid = b_worker && b_site < g.vh;
        SiteCoord bc{};
        if (b_valid) bc = coords(p.g, b_site, parity);

#pragma unroll
        for (int h0 = 0; h0 < 8; h0 += HG) {
            // ---- issue every load of this hop group (overlaps the previous tile's MMAs) ----
            uint32_t va[HG][NC], vb[HG][NC], wl[HG];
#pragma unroll
            for (int hh = 0; hh < HG; ++hh) {
                const int h = h0 + hh;
                const int mu = h >> 1;
                const bool fwd = (h & 1) == 0;
                if (row_valid) {
                    bool wrap;
                    const int64_t nb = neighbour(g, my_site, mc.xh, mc.y, mc.z, mc.t, mc.xodd, mu, fwd, &wrap);
                    const S2* psi = in + nb * site_len + rr;
                    const int pp = partner(mu, sp);
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        va[hh][c] = as_u32(psi[(int64_t)(sp * NC + c) * m]);
                        vb[hh][c] = as_u32(psi[(int64_t)(pp * NC + c) * m]);
                    }
                }
                if (b_valid) {
                    bool wrap;
                    const int64_t nb = neighbour(g, b_site, bc.xh, bc.y, bc.z, bc.t, bc.xodd, mu, fwd, &wrap);
                    uint32_t w;
                    if (fwd) {   // W = U_mu(x): (W_re, -W_im) | (W_im, W_re)
                        const uint32_t uu = as_u32(gauge[(int64_t)parity * g.vh * N2 + mu * gmu + b_site * N2 +
                                                         b_cout * NC + b_cin]);
                        w = b_riout == 0 ? (uu ^ 0x80000000u) : swap_halves(uu);
                    } else {     // W = U_mu(x-mu)^dagger: (U_re, U_im) | (-U_im, U_re)
                        const uint32_t uu = as_u32(gauge[(int64_t)(1 - parity) * g.vh * N2 + mu * gmu + nb * N2 +
                                                         b_cin * NC + b_cout]);
                        w = b_riout == 0 ? uu : (swap_halves(uu) ^ 0x00008000u);
                    }
                    if (wrap && p.t_sign < 0) w ^= 0x80008000u;
                    wl[hh] = w;
                }
            }
            // ---- first group: the previous tile's MMAs must be done before its D is read
            //      and before its A/B buffers are overwritten ----
            if (h0 == 0 && pending) {
                if (tid == 0 && !mbar_wait(&sBar, phase)) timed_out = true;
                phase ^= 1u;
                __syncthreads();
                fence_after_sync();
                epilogue(prev_site, prev_valid);
                pending = false;
            }
            // ---- A rows (TMEM) and B tiles (shared memory) of the group ----
#pragma unroll
            for (int hh = 0; hh < HG; ++hh) {
                const int h = h0 + hh;
                const int mu = h >> 1;
                const bool fwd = (h & 1) == 0;
                uint32_t av[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) av[j] = 0u;
                if (row_valid) {
                    const float cs = (fwd ? -sdag : sdag) * gsign(mu, sp);
                    const bool imag = (mu == 0 || mu == 2);
                    const P2 cvec = imag ? Pk<S>::sgn(-cs, cs) : Pk<S>::sgn(cs, cs);
                    // this row's site block starts at column col0 (0, or 4 for the second site)
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        const uint32_t ru = project(va[hh][c], vb[hh][c], imag, cvec);
                        if (NC <= 4) {
                            av[c] = col0 == 0 ? ru : 0u;
                            av[4 + c] = col0 == 0 ? 0u : ru;
                        } else {
                            av[c] = ru;
                        }
                    }
                }
                tmem_st8(tmem + lane_base + kColA + 8 * h, av);
                if (b_valid) {
                    const int n = b_sl * kb + 2 * b_cout + b_riout;
                    const int k = b_sl * kb + 2 * b_cin;
                    sB[h][b_word(n, k)] = wl[hh];
                }
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            fence_after_sync();
#pragma unroll
            for (int h = 0; h < 8; ++h)
                mma_ts(tmem + kColD, tmem + kColA + 8 * h, smem_desc(&sB[h][0], 128, 256), idesc, h > 0 ? 1u : 0u);
            mma_commit(&sBar);
        }
        pending = true;
        prev_site = my_site;
        prev_valid = row_valid;
    }
    if (pending) {
        if (tid == 0 && !mbar_wait(&sBar, phase)) timed_out = true;
        __syncthreads();
        fence_after_sync();
        epilogue(prev_site, prev_valid);
    }

    // every MMA has completed; free TMEM
    fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        fence_after_sync();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                     : "memory");
    }
    if (timed_out && err != nullptr) atomicExch(err, 1);

    if constexpr (NV > 0) {
        // per-RHS block sums in a fixed order: rows with the same RHS r, in row order
#pragma unroll
        for (int k = 0; k < NV; ++k) sRow[k * kThreads + tid] = row_used ? red[k] : make_double2(0.0, 0.0);
        __syncthreads();
        for (int idx = tid; idx < NV * m; idx += kThreads) {
            const int k = idx / m, j = idx - k * m;
            double2 s = make_double2(0.0, 0.0);
            for (int i = 0; i < kThreads; ++i) {
                const int w = i % rows_site;
                if (i / rows_site < spt && w % m == j) {
                    s.x += sRow[k * kThreads + i].x;
                    s.y += sRow[k * kThreads + i].y;
                }
            }
            sRed[idx] = s;
        }
        __syncthreads();
        publish_and_finish<NV>(sRed, m, p.red);
    }
}

template <int NC, typename S>
int launch_tc(const HopParams& p, bool dagger, int epi, cudaStream_t st) {
    void (*k)(const HopParams, int*) = nullptr;
    switch (epi) {
        case EPI_PLAIN: k = dagger ? hop_tc_kernel<NC, S, true, EPI_PLAIN> : hop_tc_kernel<NC, S, false, EPI_PLAIN>; break;
        case EPI_XPAY: k = dagger ? hop_tc_kernel<NC, S, true, EPI_XPAY> : hop_tc_kernel<NC, S, false, EPI_XPAY>; break;
        case EPI_SCHUR_R0: k = hop_tc_kernel<NC, S, false, EPI_SCHUR_R0>; break;
        case EPI_SCHUR_TS: k = hop_tc_kernel<NC, S, false, EPI_SCHUR_TS>; break;
        case EPI_SCHUR: k = hop_tc_kernel<NC, S, false, EPI_SCHUR>; break;
        case EPI_RESID: k = hop_tc_kernel<NC, S, false, EPI_RESID>; break;
        default: return set_error(QCU_ERR_INVALID, "unknown hop epilogue %d", epi);
    }
    if (dagger && epi != EPI_PLAIN && epi != EPI_XPAY)
        return set_error(QCU_ERR_UNSUPPORTED, "dagger hop only with plain/xpay epilogue");
    const int rows_site = 4 * p.m;
    const int spt = (rows_site <= 64 && 2 * NC <= 8) ? 2 : 1;
    const int64_t ntiles = (p.g.vh + spt - 1) / spt;
    int per_sm = blocks_per_sm(reinterpret_cast<const void*>(k), kThreads);
    if (per_sm <= 1) {   // occupancy query unavailable: estimate from the register count
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, k) == cudaSuccess && fa.numRegs > 0)
            per_sm = 65536 / (((fa.numRegs + 7) / 8 * 8) * kThreads);
        cudaGetLastError();
    }
    // at most 512 / kTmemCols CTAs per SM can hold their TMEM allocation at once
    const int tmem_cap = 512 / kTmemCols;
    if (per_sm > tmem_cap) per_sm = tmem_cap;
    if (per_sm < 1) per_sm = 1;
    const int64_t cap = (int64_t)per_sm * sm_count();
    int grid = (int)(ntiles < cap ? ntiles : cap);
    if (grid > kScratchBlocks) grid = kScratchBlocks;
    if (grid < 1) grid = 1;
    k<<<grid, kThreads, 0, st>>>(p, device_error_flag());
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

}  // namespace tc

// Tensor-core hop for FP16/BF16 storage: n_color 2..8 with 2*n_color*sites_per_tile <= 16
// and 4*m <= 128.  Returns QCU_ERR_UNSUPPORTED for shapes it does not cover.
bool hop_tc_supported(int nc, int m, int prec) {
    if (prec != QCU_PRECISION_HALF && prec != QCU_PRECISION_BF16) return false;
    if (nc < 2 || nc > 8) return false;
    return 4 * m <= 128;
}

int hop_tc_launch(const HopParams& p, int nc, int prec, bool dagger, int epi, cudaStream_t st) {
    if (!hop_tc_supported(nc, p.m, prec))
        return set_error(QCU_ERR_UNSUPPORTED, "tensor-core hop: n_color=%d m=%d precision=%d", nc, p.m, prec);
    auto go = [&](auto tag) -> int {
        using S = decltype(tag);
        switch (nc) {
            case 2: return tc::launch_tc<2, S>(p, dagger, epi, st);
            case 3: return tc::launch_tc<3, S>(p, dagger, epi, st);
            case 4: return tc::launch_tc<4, S>(p, dagger, epi, st);
            case 5: return tc::launch_tc<5, S>(p, dagger, epi, st);
            case 6: return tc::launch_tc<6, S>(p, dagger, epi, st);
            case 7: return tc::launch_tc<7, S>(p, dagger, epi, st);
            default: return tc::launch_tc<8, S>(p, dagger, epi, st);
        }
    };
    if (prec == QCU_PRECISION_HALF) return go(__half{});
    return go(__nv_bfloat16{});
}

}  // namespace qcub
