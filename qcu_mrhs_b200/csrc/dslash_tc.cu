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

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Bounded wait for the phase with the given parity to complete: gives up after ~2^30 SM
// cycles (about half a second) and returns false.  Callers stop waiting once a wait has
// failed, so a kernel whose pipeline broke finishes quickly with its error flag set.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t addr = smem_u32(bar);
    const long long t0 = clock64();
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(addr), "r"(parity)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > (1ll << 30)) return false;
    }
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

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// bulk global -> shared copy completing on an mbarrier (16-byte aligned, size % 16 == 0)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

__device__ __forceinline__ void tmem_st4(uint32_t taddr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr), "r"(a), "r"(b),
                 "r"(c), "r"(d)
                 : "memory");
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[16]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr)
                 : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
#pragma unroll
    for (int i = 8; i < 16; ++i) v[i] = 0.f;
}

constexpr int kStages = 3;
constexpr int kCTA = 160;       // 4 consumer warps (TMEM lanes 0..127) + 1 producer warp

// Shared-memory plan (32-bit words): kStages x { spinors [spt][8 hops][site_len],
// links [spt][8 hops][N*N] }, then 8 B tiles of 128 words.
struct TcPlan {
    int spt, rows_block, site_len, stage_words, link_off;
};
__host__ __device__ inline TcPlan tc_plan(int nc, int m) {
    TcPlan q;
    q.spt = (4 * m <= 64 && 2 * nc <= 8) ? 2 : 1;
    q.rows_block = q.spt == 2 ? 64 : 128;
    q.site_len = 4 * nc * m;
    q.link_off = q.spt * 8 * q.site_len;
    q.stage_words = q.link_off + q.spt * 8 * nc * nc;
    q.stage_words = (q.stage_words + 31) & ~31;   // keep every stage 128-byte aligned
    return q;
}
inline size_t tc_smem_bytes(int nc, int m) {
    const TcPlan q = tc_plan(nc, m);
    return (size_t)(kStages * q.stage_words + 8 * 128) * 4;
}

template <int NC, typename S, bool DAG, int EPI>
__global__ void __launch_bounds__(kCTA, 3) hop_tc_kernel(const HopParams p, int* err) {
    using S2 = typename St<S>::S2;
    using A2 = typename St<S>::A2;
    using P2 = typename Pk<S>::T2;
    constexpr int NV = (EPI == EPI_SCHUR_R0 || EPI == EPI_RESID) ? 1 : (EPI == EPI_SCHUR_TS ? 2 : 0);
    constexpr int N2 = NC * NC;
    extern __shared__ __align__(128) uint32_t smem[];
    __shared__ __align__(8) uint64_t sFull[kStages];
    __shared__ __align__(8) uint64_t sEmpty[kStages];
    __shared__ __align__(8) uint64_t sMma;
    __shared__ uint32_t sTmem;
    __shared__ double2 sRed[NV > 0 ? NV * kMaxRhs : 1];
    __shared__ double2 sRow[NV > 0 ? NV * 128 : 1];

    if (skip_launch(p.done, p.gate)) return;
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int m = p.m;
    const TcPlan plan = tc_plan(NC, m);
    const int spt = plan.spt;
    const int site_len = plan.site_len;
    const int64_t vh = p.g.vh;
    const int64_t ntiles = (vh + spt - 1) / spt;
    const int parity = p.parity;
    uint32_t* sB = smem + kStages * plan.stage_words;

    // ---- one-time set-up ----
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&sFull[s], 1 + spt * 8);   // producer's expect_tx + one per staged link
            mbar_init(&sEmpty[s], 128);          // every consumer thread releases the stage
        }
        mbar_init(&sMma, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < 8 * 128; i += kCTA) sB[i] = 0u;
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
    bool timed_out = false;

    if (warp == 4) {
        // ================= producer warp: stage neighbour spinors and links =================
        const S2* __restrict__ in = static_cast<const S2*>(p.in);
        const uint32_t* __restrict__ gauge = static_cast<const uint32_t*>(p.gauge);
        const int64_t gmu = 2 * vh * N2;
        const uint32_t site_bytes = (uint32_t)site_len * 4u;
        int64_t it = 0;
        for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
            const int stage = (int)(it % kStages);
            if (it >= kStages && !timed_out) {
                if (!mbar_wait(&sEmpty[stage], (uint32_t)((it / kStages) - 1) & 1u)) timed_out = true;
            }
            uint32_t* st = smem + stage * plan.stage_words;
            const int64_t site0 = tile * spt;
            const int nvalid = (int)((vh - site0) < spt ? (vh - site0) : spt);
            if (lane == 0) mbar_arrive_tx(&sFull[stage], (uint32_t)nvalid * 8u * site_bytes);
            __syncwarp();
            if (lane < spt * 8) {
                const int sl = lane >> 3, h = lane & 7, mu = h >> 1;
                const bool fwd = (h & 1) == 0;
                const int64_t site = site0 + sl;
                if (sl < nvalid) {
                    const SiteCoord c = coords(p.g, site, parity);
                    bool wrap;
                    const Tile tg{p.g.lxh, p.g.L[1], p.g.L[2], p.g.L[3], vh};
                    const int64_t nb = neighbour(tg, site, c.xh, c.y, c.z, c.t, c.xodd, mu, fwd, &wrap);
                    bulk_g2s(st + (sl * 8 + h) * site_len, in + nb * site_len, site_bytes, &sFull[stage]);
                    const uint32_t* U = fwd ? gauge + (int64_t)parity * vh * N2 + mu * gmu + site * N2
                                            : gauge + (int64_t)(1 - parity) * vh * N2 + mu * gmu + nb * N2;
                    const uint32_t flip = (wrap && p.t_sign < 0) ? 0x80008000u : 0u;
                    uint32_t* dl = st + plan.link_off + (sl * 8 + h) * N2;
#pragma unroll
                    for (int e = 0; e < N2; ++e) dl[e] = __ldg(U + e) ^ flip;
                }
                mbar_arrive(&sFull[stage]);   // release: the link words above are visible to consumers
            }
        }
        // drain: every bulk copy this CTA issued has landed before the CTA can exit (bounded;
        // in a healthy run the consumers already waited on all of these phases)
        if (lane == 0) {
            for (int64_t k = (it > kStages ? it - kStages : 0); k < it; ++k)
                if (!mbar_wait(&sFull[(int)(k % kStages)], (uint32_t)(k / kStages) & 1u)) timed_out = true;
        }
    } else {
        // ================= consumer warps: A rows (TMEM), B tiles, MMA, epilogue =================
        const int rows_block = plan.rows_block;
        const int sl = tid / rows_block;
        const int within = tid - sl * rows_block;
        const bool row_used = sl < spt && within < 4 * m;
        const int sp = row_used ? within / m : 0;
        const int rr = row_used ? within - sp * m : 0;
        const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
        const uint32_t idesc = instr_desc(Pk<S>::fmt);
        const int kb = spt == 2 ? 8 : 16;
        // projection coefficient per hop: 1 + sigma gamma_mu, sigma = -s forward, +s backward
        P2 cvec[8];
#pragma unroll
        for (int h = 0; h < 8; ++h) {
            const int mu = h >> 1;
            const float cs = ((h & 1) == 0 ? (DAG ? 1.f : -1.f) : (DAG ? -1.f : 1.f)) * gsign(mu, sp);
            cvec[h] = (mu == 0 || mu == 2) ? Pk<S>::sgn(-cs, cs) : Pk<S>::sgn(cs, cs);
        }
        const int pp_lo = partner(0, sp), pp_hi = partner(2, sp);   // partner for mu < 2, mu >= 2
        // B work item: (site block, c_out, ri_out, c_in)
        const bool b_worker = tid < spt * NC * 2 * NC;
        int b_sl = 0, b_cout = 0, b_riout = 0, b_cin = 0;
        if (b_worker) {
            int q = tid;
            b_cin = q % NC; q /= NC;
            b_riout = q % 2; q /= 2;
            b_cout = q % NC;
            b_sl = q / NC;
        }
        const int b_word_idx = b_worker ? b_word(b_sl * kb + 2 * b_cout + b_riout, b_sl * kb + 2 * b_cin) : 0;

        // zero this row's A columns once (the other site's block and padding stay zero)
#pragma unroll
        for (int h = 0; h < 8; ++h) tmem_st4(tmem + lane_base + kColA + 8 * h, 0u, 0u, 0u, 0u),
                                    tmem_st4(tmem + lane_base + kColA + 8 * h + 4, 0u, 0u, 0u, 0u);

        double2 red[NV > 0 ? NV : 1];
#pragma unroll
        for (int k = 0; k < (NV > 0 ? NV : 1); ++k) red[k] = make_double2(0.0, 0.0);

        auto epilogue = [&](int64_t site, bool valid) {
            float d[16];
            if (spt == 2) tmem_ld8(tmem + lane_base + kColD + 8 * sl, d);
            else tmem_ld16(tmem + lane_base + kColD, d);
            fence_before_sync();
            if (!valid) return;
            S2* __restrict__ out = static_cast<S2*>(p.out);
            const S2* __restrict__ xv = static_cast<const S2*>(p.x);
            const S2* __restrict__ r0v = static_cast<const S2*>(p.r0);
            const int64_t base = site * site_len + rr;
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const int64_t o = base + (int64_t)(sp * NC + c) * m;
                const A2 v = mk2<A2>(d[2 * c], d[2 * c + 1]);
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

        uint32_t mma_phase = 0;
        bool pending = false;
        int64_t prev_site = 0;
        bool prev_valid = false;
        int64_t it = 0;
        for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
            const int stage = (int)(it % kStages);
            if (!timed_out && !mbar_wait(&sFull[stage], (uint32_t)(it / kStages) & 1u)) timed_out = true;
            const uint32_t* st = smem + stage * plan.stage_words;
            const int64_t my_site = tile * spt + sl;
            const bool row_valid = row_used && my_site < vh;
            // ---- operands of the 8 hops from the staged tile ----
            uint32_t va[8][NC], vb[8][NC], wl[8];
            const uint32_t* rowp = st + sl * 8 * site_len + rr;
#pragma unroll
            for (int h = 0; h < 8; ++h) {
                const int pp = (h >> 1) < 2 ? pp_lo : pp_hi;
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    va[h][c] = row_valid ? rowp[h * site_len + (sp * NC + c) * m] : 0u;
                    vb[h][c] = row_valid ? rowp[h * site_len + (pp * NC + c) * m] : 0u;
                }
                if (b_worker) {
                    const bool fwd = (h & 1) == 0;
                    const uint32_t uu =
                        st[plan.link_off + (b_sl * 8 + h) * N2 + (fwd ? b_cout * NC + b_cin : b_cin * NC + b_cout)];
                    // forward W = U: (W_re,-W_im) | (W_im,W_re); backward W = U^dag: (U_re,U_im) | (-U_im,U_re)
                    wl[h] = fwd ? (b_riout == 0 ? (uu ^ 0x80000000u) : swap_halves(uu))
                                : (b_riout == 0 ? uu : (swap_halves(uu) ^ 0x00008000u));
                }
            }
            mbar_arrive(&sEmpty[stage]);   // stage consumed (values are in registers)
            // ---- previous tile: MMAs done -> epilogue; frees D, A and B ----
            if (pending) {
                if (tid == 0 && !timed_out && !mbar_wait(&sMma, mma_phase)) timed_out = true;
                mma_phase ^= 1u;
                consumer_sync();
                fence_after_sync();
                epilogue(prev_site, prev_valid);
            }
            // ---- A rows and B tiles ----
#pragma unroll
            for (int h = 0; h < 8; ++h) {
                const bool imag = ((h >> 1) == 0 || (h >> 1) == 2);
                uint32_t r[NC];
#pragma unroll
                for (int c = 0; c < NC; ++c) r[c] = project(va[h][c], vb[h][c], imag, cvec[h]);
                if (spt == 2) {
                    tmem_st4(tmem + lane_base + kColA + 8 * h + 4 * sl, r[0], NC > 1 ? r[NC > 1 ? 1 : 0] : 0u,
                             NC > 2 ? r[NC > 2 ? 2 : 0] : 0u, NC > 3 ? r[NC > 3 ? 3 : 0] : 0u);
                } else {
                    uint32_t av[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) av[j] = j < NC ? r[j < NC ? j : 0] : 0u;
                    tmem_st8(tmem + lane_base + kColA + 8 * h, av);
                }
                if (b_worker) sB[h * 128 + b_word_idx] = wl[h];
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            fence_before_sync();
            consumer_sync();
            if (tid == 0) {
                fence_after_sync();
#pragma unroll
                for (int h = 0; h < 8; ++h)
                    mma_ts(tmem + kColD, tmem + kColA + 8 * h, smem_desc(sB + h * 128, 128, 256), idesc,
                           h > 0 ? 1u : 0u);
                mma_commit(&sMma);
            }
            pending = true;
            prev_site = my_site;
            prev_valid = row_valid;
        }
        if (pending) {   // always wait (bounded) for the last MMAs before TMEM is freed
            if (tid == 0 && !mbar_wait(&sMma, mma_phase)) timed_out = true;
            consumer_sync();
            fence_after_sync();
            epilogue(prev_site, prev_valid);
        }
        if constexpr (NV > 0) {
#pragma unroll
            for (int k = 0; k < NV; ++k) sRow[k * 128 + tid] = row_used ? red[k] : make_double2(0.0, 0.0);
        }
    }

    // all MMAs have completed and every stage has been consumed; free TMEM
    fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        fence_after_sync();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                     : "memory");
    }
    if (timed_out && err != nullptr) atomicExch(err, 1);

    if constexpr (NV > 0) {
        // per-RHS block sums in a fixed order: rows of the same RHS, in row order
        const int rows_block = plan.rows_block;
        for (int idx = tid; idx < NV * m; idx += kCTA) {
            const int k = idx / m, j = idx - k * m;
            double2 s = make_double2(0.0, 0.0);
            for (int i = 0; i < 128; ++i) {
                const int bsl = i / rows_block, w = i - bsl * rows_block;
                if (bsl < spt && w < 4 * m && w % m == j) {
                    s.x += sRow[k * 128 + i].x;
                    s.y += sRow[k * 128 + i].y;
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
    const size_t smem = tc_smem_bytes(NC, p.m);
    static bool attr_set[2][6] = {};
    const int di = dagger ? 1 : 0;
    if (!attr_set[di][epi]) {
        QCUB_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        attr_set[di][epi] = true;
    }
    const TcPlan plan = tc_plan(NC, p.m);
    const int64_t ntiles = (p.g.vh + plan.spt - 1) / plan.spt;
    int per_sm = blocks_per_sm(reinterpret_cast<const void*>(k), kCTA, smem);
    if (per_sm <= 1) {   // occupancy query unavailable: estimate from the register count
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, k) == cudaSuccess && fa.numRegs > 0)
            per_sm = 65536 / (((fa.numRegs + 7) / 8 * 8) * kCTA);
        cudaGetLastError();
    }
    const int tmem_cap = 512 / kTmemCols;   // CTAs per SM that can hold their TMEM at once
    if (per_sm > tmem_cap) per_sm = tmem_cap;
    if (per_sm < 1) per_sm = 1;
    const int64_t cap = (int64_t)per_sm * sm_count();
    int grid = (int)(ntiles < cap ? ntiles : cap);
    if (grid > kScratchBlocks) grid = kScratchBlocks;
    if (grid < 1) grid = 1;
    k<<<grid, kCTA, smem, st>>>(p, device_error_flag());
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

}  // namespace tc

// Tensor-core hop for FP16/BF16 storage: n_color 2..4 and 4*m <= 128, input 16-byte aligned.
// Returns QCU_ERR_UNSUPPORTED for shapes it does not cover.
bool hop_tc_supported(int nc, int m, int prec) {
    if (prec != QCU_PRECISION_HALF && prec != QCU_PRECISION_BF16) return false;
    if (nc < 2 || nc > 4) return false;   // operands of 8 hops are held in registers
    return 4 * m <= 128;
}

int hop_tc_launch(const HopParams& p, int nc, int prec, bool dagger, int epi, cudaStream_t st) {
    if (reinterpret_cast<uintptr_t>(p.in) % 16 != 0)
        return set_error(QCU_ERR_UNSUPPORTED, "tensor-core hop: input spinor not 16-byte aligned");
    if (!hop_tc_supported(nc, p.m, prec))
        return set_error(QCU_ERR_UNSUPPORTED, "tensor-core hop: n_color=%d m=%d precision=%d", nc, p.m, prec);
    auto go = [&](auto tag) -> int {
        using S = decltype(tag);
        switch (nc) {
            case 2: return tc::launch_tc<2, S>(p, dagger, epi, st);
            case 3: return tc::launch_tc<3, S>(p, dagger, epi, st);
            default: return tc::launch_tc<4, S>(p, dagger, epi, st);
        }
    };
    if (prec == QCU_PRECISION_HALF) return go(__half{});
    return go(__nv_bfloat16{});
}

}  // namespace qcub
