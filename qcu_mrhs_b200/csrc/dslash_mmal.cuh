// dslash_mmal.cuh -- fragment helpers shared by the link-operand tensor-core hop kernels
// (dslash_mmal.cu: N <= 4; dslash_mmal_big.cu: 5 <= N <= 8).
//
// MMA (mma.sync m16n8k16, 16-bit operands, FP32 accumulation) with the LINKS as the A operand
// and the projected neighbour spinors as the B operand.
//
// Same operator, layouts and epilogues as dslash_impl.cuh (reference
// include/kernel/su_n_m_rhs_dslash.cuh:92-105, complex_matmul.cuh:16-600, whose solver hop
// also runs the link products through tensor-core tiles).
//
// Work unit: one warp per (half-site, chunk of up to 16 RHS); inside it, groups of 4 RHS.
// For direction mu, with the forward hop matrix W_f = U_mu(x) (t-boundary sign folded in)
// and the backward one W_b = U_mu(x - mu)^dag, one real MMA per group of 4 RHS does both hops:
//   K (16)   8 complex slots as (re, im) pairs: slot c = forward colour c, slot 4 + c =
//            backward colour c (N <= 4; the rest zero)
//   B (16x8) column j = (RHS j/2 of the group, half spinor j%2): the projected forward and
//            backward neighbour half spinors h_f, h_b (lane 4g+t holds column g, colour t)
//   A (16x16) rows 0..2N-1, "sum" rows (c', re/im):  [emb(W_f)      | emb(W_b)]
//            rows 8..8+2N-1, "diff" rows (c', re/im): [emb(phi W_f) | emb(-phi W_b)]
//   D        sum rows: W_f h_f + W_b h_b, which spins 0 and 1 take as they are (column
//            h = 0 and 1); diff rows: phi (W_f h_f - W_b h_b), phi = the lower-spin phase of
//            the forward projector (the backward projector's is -phi)
// emb(W) is the real embedding [[W.re, -W.im], [W.im, W.re]] of each complex entry.  The
// lower spins take the diff rows with a direction-dependent column (the x and y projectors
// exchange the half spinors) and sign (y and z flip spin 3), so every direction has its
// own D tile (4 FP32 per lane) and the tiles are added at the end, in FP32:
//   spin0 = sum_mu D_mu[sum, h0]          spin1 = sum_mu D_mu[sum, h1]
//   spin2 = D_x[diff,h1] + D_y[diff,h1] + D_z[diff,h0] + D_t[diff,h0]
//   spin3 = D_x[diff,h0] - D_y[diff,h0] - D_z[diff,h1] + D_t[diff,h1]
// So the link products and all sums are FP32; the only 16-bit arithmetic is the spin
// projection (one rounding of p_a + kappa p_b, kappa in {+-1, +-i}) and the final store.
//
// Fragment layouts (PTX ISA, mma.m16n8k16, 16-bit A/B): lane = 4 g + t holds
//   A: a0 = (row g, k 2t..2t+1), a1 = (row g+8, k 2t..), a2 = (row g, k 2t+8..), a3 = (row g+8, k 2t+8..)
//   B: b0 = (k 2t..2t+1, col g), b1 = (k 2t+8..2t+9, col g)
//   D: d0, d1 = (row g, col 2t..2t+1), d2, d3 = (row g+8, col 2t..2t+1)
// so lane (g, t) builds its A words from the link elements W_f[g/2][t], W_b[g/2][t], loads
// the neighbour words of (half spinor g%2, colour t, RHS g/2) and ends with component g%2
// (re/im) of the four output spins of (colour g/2, RHS t).  Lanes g and g^1 (lane ^ 4)
// exchange halves so that each stores two whole complex words.  Lanes outside the colour
// range load clamped (finite) words that meet zero A entries, and store nothing.
//
// For 5 <= N <= 8 the sum and diff rows are two M tiles and the forward and backward
// colours two K steps (4 MMAs per direction and group); the sum tile is shared by the
// directions, the diff tiles are per direction.
#pragma once

#include <type_traits>

#include "dslash.h"
#include "dslash_impl.cuh"
#include "workspace.h"

namespace qcub {

int* device_error_flag();   // runtime.cu: per-device flag, nonzero after a timed-out wait

// the hop for 5 <= N <= 8 (dslash_mmal_big.cu)
int hop_mmal_big_launch(const HopParams& p, int nc, int prec, bool dagger, int epi, cudaStream_t st);

namespace {

constexpr int kLThreads = 256;
constexpr int kLWarps = kLThreads / 32;
constexpr int kLMaxChunkRhs = 16;   // RHS per work unit (4 groups of 4)

template <typename S> struct LMma;
template <> struct LMma<__half> {
    static constexpr uint32_t kOne = 0x3C00u;
    __device__ static void mma(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1, float c0,
                               float c1, float c2, float c3) {
        asm("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%10,%11,%12,%13};"
            : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
            : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1), "f"(c0), "f"(c1), "f"(c2), "f"(c3));
    }
    __device__ static uint32_t fma(uint32_t a, uint32_t b, uint32_t c) {
        const __half2 r = __hfma2(*reinterpret_cast<const __half2*>(&a), *reinterpret_cast<const __half2*>(&b),
                                  *reinterpret_cast<const __half2*>(&c));
        return *reinterpret_cast<const uint32_t*>(&r);
    }
    __device__ static uint32_t pack(float lo, float hi) {
        const __half2 r = __floats2half2_rn(lo, hi);
        return *reinterpret_cast<const uint32_t*>(&r);
    }
    __device__ static float2 unpack(uint32_t u) { return __half22float2(*reinterpret_cast<const __half2*>(&u)); }
};
template <> struct LMma<__nv_bfloat16> {
    static constexpr uint32_t kOne = 0x3F80u;
    __device__ static void mma(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1, float c0,
                               float c1, float c2, float c3) {
        asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%10,%11,%12,%13};"
            : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
            : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1), "f"(c0), "f"(c1), "f"(c2), "f"(c3));
    }
    __device__ static uint32_t fma(uint32_t a, uint32_t b, uint32_t c) {
        const __nv_bfloat162 r = __hfma2(*reinterpret_cast<const __nv_bfloat162*>(&a),
                                         *reinterpret_cast<const __nv_bfloat162*>(&b),
                                         *reinterpret_cast<const __nv_bfloat162*>(&c));
        return *reinterpret_cast<const uint32_t*>(&r);
    }
    __device__ static uint32_t pack(float lo, float hi) {
        const __nv_bfloat162 r = __floats2bfloat162_rn(lo, hi);
        return *reinterpret_cast<const uint32_t*>(&r);
    }
    __device__ static float2 unpack(uint32_t u) {
        return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u));
    }
};

// packed pair of +-1 in the 16-bit format (lo in the low half)
template <typename S>
__host__ __device__ constexpr uint32_t unit_pair(int lo, int hi) {
    return (LMma<S>::kOne | (lo < 0 ? 0x8000u : 0u)) | ((LMma<S>::kOne | (hi < 0 ? 0x8000u : 0u)) << 16);
}
__device__ __forceinline__ uint32_t swap_halves(uint32_t u) { return __byte_perm(u, 0, 0x1032); }

// phase codes: 0 = +1, 1 = -1, 2 = +i, 3 = -i
__host__ __device__ constexpr int lphase(int s, bool imag) { return (imag ? 2 : 0) + (s > 0 ? 0 : 1); }
// lower-spin phase of spin 2 for direction MU and projector sign SG (spin2 += C2 (W h)_{P2});
// spin 3 takes +-C2 (W h)_{P3} (the tables of dslash_impl.cuh)
template <int MU, int SG>
struct LRecon {
    static constexpr int C2 = MU == 0 ? lphase(-SG, true) : MU == 1 ? lphase(SG, false)
                            : MU == 2 ? lphase(-SG, true) : lphase(SG, false);
};
// emb(c W) from e = emb(W) of this lane's row (re rows: (W.re, -W.im), im rows: (W.im, W.re)):
//   emb(-W) = e ^ sign bits; emb(iW) = swap(e) ^ high sign; emb(-iW) = swap(e) ^ low sign
template <int C>
__device__ __forceinline__ uint32_t emb_phase(uint32_t e) {
    if (C == 0) return e;
    if (C == 1) return e ^ 0x80008000u;
    if (C == 2) return swap_halves(e) ^ 0x80000000u;
    return swap_halves(e) ^ 0x00008000u;
}

// Projection of one neighbour word pair for lane column h = g % 2 (see the kernel comment):
//   MU 0: h = p_h + s i p_{3-h}      MU 1: h = p_h + (h ? s : -s) p_{3-h}
//   MU 2: h = p_h + (h ? -s : s) i p_{2+h}      MU 3: h = p_h + s p_{2+h}
// as one packed FMA p + mult * q (q swapped for the i cases); `lm` is the lane's multiplier
// for MU 1 / MU 2 (it depends on h).
template <typename S, int MU, int SG>
__device__ __forceinline__ uint32_t lproject(uint32_t pw, uint32_t qw, uint32_t lm) {
    using M = LMma<S>;
    if (MU == 0) return M::fma(swap_halves(qw), unit_pair<S>(-SG, SG), pw);
    if (MU == 1) return M::fma(qw, lm, pw);
    if (MU == 2) return M::fma(swap_halves(qw), lm, pw);
    return M::fma(qw, unit_pair<S>(SG, SG), pw);
}

// Groups of 4 RHS (the 4 B columns pairs of one MMA) that a work unit computes: bit n for
// group n (RHS rb0 + 4n .. rb0 + 4n + 3) if it holds an RHS below m and, when per-RHS
// activity flags are given, at least one active RHS.  Warp-uniform.
template <int NTC>
__device__ __forceinline__ uint32_t active_groups(const int* __restrict__ active, int rb0, int m) {
    uint32_t gm = 0u;
#pragma unroll
    for (int n = 0; n < NTC; ++n) {
        const int r0 = rb0 + 4 * n;
        if (r0 >= m) break;
        bool on = active == nullptr;
#pragma unroll
        for (int r = 0; r < 4; ++r)
            if (!on && r0 + r < m) on = __ldg(active + r0 + r) != 0;
        if (on) gm |= 1u << n;
    }
    return gm;
}

// A fragment of direction MU.  Rows are ordered (re/im, sum/diff, colour): lane (g, t) holds
// rows g (re) and g + 8 (im) of class cls = g / 4 (0 sum, 1 diff) and colour g % 4, for
// K slots t (forward colour t) and t + 4 (backward colour t).  wf = W_f[g%4][t] (t-boundary
// sign folded in), wb = W_b[g%4][t] = conj(U_b[t][g%4]); diff lanes take phi W_f and -phi W_b,
// applied as a lane byte permute (psel: identity or half swap) and sign mask (pmf / pmb).
// emb re row: (w.re, -w.im) = w ^ high sign; im row: (w.im, w.re) = swap(w).
__device__ __forceinline__ void mmal_a(uint32_t (&A)[4], uint32_t wf, uint32_t wb, uint32_t okm, uint32_t psel,
                                       uint32_t pmf, uint32_t pmb) {
    const uint32_t ff = (__byte_perm(wf, 0, psel) ^ pmf) & okm;
    const uint32_t fb = (__byte_perm(wb, 0, psel) ^ pmb) & okm;
    A[0] = ff ^ 0x80000000u;
    A[1] = swap_halves(ff);
    A[2] = fb ^ 0x80000000u;
    A[3] = swap_halves(fb);
}

// lane phase constants of the diff rows for a direction whose forward lower-spin phase has
// code C (0 = +1, 1 = -1, 2 = +i, 3 = -i): phi w = perm(w, sel) ^ mask (i w = swap(w) ^ low sign)
struct LPhase {
    uint32_t sel, mf, mb;
};
template <int C>
__device__ __forceinline__ LPhase lphase_lane(bool diff) {
    LPhase r;
    constexpr bool imag = C >= 2;
    constexpr uint32_t mpos = imag ? 0x00008000u : 0u;              // +1 or +i
    constexpr uint32_t mneg = imag ? 0x80000000u : 0x80008000u;     // -1 or -i
    constexpr bool neg = (C & 1) != 0;
    r.sel = (diff && imag) ? 0x1032u : 0x3210u;
    r.mf = diff ? (neg ? mneg : mpos) : 0u;
    r.mb = diff ? (neg ? mpos : mneg) : 0u;   // backward: -phi
    return r;
}

}  // namespace
}  // namespace qcub
