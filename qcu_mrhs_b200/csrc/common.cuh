// common.cuh -- shared types for the B200 multi-RHS Wilson library.
//
// Precision codes follow the reference's QcuPrecision order (half, single, double,
// undefined); the numeric values live in an external header that is not part of
// the reference tree, so these are this library's choice.  BF16 is an extension.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/qcu_b200.h"

namespace qcub {

constexpr int kNs = 4;          // spin components
constexpr int kNd = 4;          // space-time dimensions
constexpr int kMaxColor = 8;    // largest N with a compiled kernel
constexpr int kMaxRhs = 64;     // largest m (per call) supported by the kernels
// Site-blocked spinor layout (the mixed solver's 16-bit vectors): blocks of kSiteBlock
// half-lattice sites; inside a block the 4N spin-colour rows one after another, each row
// holding the block's sites with their m right-hand sides innermost:
//   complex (site n, row r, RHS j) at ((n / kSiteBlock) 4N + r) kSiteBlock m + (n % kSiteBlock) m + j.
// A warp's load of one row of consecutive sites is then one contiguous run.
constexpr int kSiteBlock = 32;

// Site-blocked complex index of gathered index gi = (site rows + row) m + j, rows = 4N
// (fewer than 2^31 complex in all).
__device__ __forceinline__ int64_t site_blocked_index(int64_t gi, int m, int rows) {
    const uint32_t g = (uint32_t)gi, um = (uint32_t)m, ur = (uint32_t)rows;
    const uint32_t q = g / um, j = g - q * um;
    const uint32_t n = q / ur, r = q - n * ur;
    const uint32_t b = n / kSiteBlock, ns = n - b * kSiteBlock;
    return ((int64_t)(b * ur + r) * kSiteBlock + ns) * um + j;
}

// Record an error for qcuGetLastStatus()/qcuGetLastError(); returns the status.
int set_error(int status, const char* fmt, ...);
void clear_error();

#define QCUB_CUDA_CHECK(expr)                                                                 \
    do {                                                                                      \
        cudaError_t _e = (expr);                                                              \
        if (_e != cudaSuccess)                                                                \
            return ::qcub::set_error(QCU_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #expr,   \
                                     cudaGetErrorString(_e));                                 \
    } while (0)

#define QCUB_CHECK_LAUNCH() QCUB_CUDA_CHECK(cudaGetLastError())

// Division by a fixed divisor d (1 <= d < 2^31) of n < 2^31 with one multiply-high:
// q = (umulhi(n, m) + n) >> l with l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1
// (round-up reciprocal method); (umulhi(n, m) + n) < 2^32 because both terms are < 2^31.
struct FastDiv {
    uint32_t d = 1, m = 1, l = 0;
    __host__ __device__ __forceinline__ uint32_t div(uint32_t n) const {
#ifdef __CUDA_ARCH__
        return (__umulhi(n, m) + n) >> l;
#else
        return (uint32_t)((((uint64_t)n * m) >> 32) + n) >> l;
#endif
    }
};

inline FastDiv make_fastdiv(uint32_t d) {
    FastDiv f;
    f.d = d;
    uint32_t l = 0;
    while (l < 31 && (1ull << l) < d) ++l;
    f.l = l;
    f.m = (uint32_t)((((1ull << 32) * ((1ull << l) - d)) / d + 1) & 0xFFFFFFFFull);
    return f;
}

// Lattice geometry of one process (single GPU: the whole lattice).
struct Geom {
    int L[4];      // Lx, Ly, Lz, Lt
    int lxh;       // Lx / 2
    int64_t vh;    // half volume (< 2^31: half-site indices are 32-bit in the kernels)
    FastDiv dx, dy, dz;   // division by Lx/2, Ly, Lz
};

inline Geom make_geom(const int L[4]) {
    Geom g;
    for (int i = 0; i < 4; ++i) g.L[i] = L[i];
    g.lxh = L[0] / 2;
    g.vh = (int64_t)L[0] * L[1] * L[2] * L[3] / 2;
    g.dx = make_fastdiv((uint32_t)(g.lxh > 0 ? g.lxh : 1));
    g.dy = make_fastdiv((uint32_t)(L[1] > 0 ? L[1] : 1));
    g.dz = make_fastdiv((uint32_t)(L[2] > 0 ? L[2] : 1));
    return g;
}

// half-site index -> (xh, y, z, t) with three multiply-high divisions
struct SiteXYZT {
    int xh, y, z, t;
};
__host__ __device__ __forceinline__ SiteXYZT site_coords(const Geom& g, uint32_t site) {
    SiteXYZT c;
    const uint32_t q1 = g.dx.div(site);
    c.xh = (int)(site - q1 * (uint32_t)g.lxh);
    const uint32_t q2 = g.dy.div(q1);
    c.y = (int)(q1 - q2 * (uint32_t)g.L[1]);
    const uint32_t q3 = g.dz.div(q2);
    c.z = (int)(q2 - q3 * (uint32_t)g.L[2]);
    c.t = (int)q3;
    return c;
}

inline size_t prec_bytes(int prec) {  // bytes of one real number
    switch (prec) {
        case QCU_PRECISION_DOUBLE: return 8;
        case QCU_PRECISION_SINGLE: return 4;
        case QCU_PRECISION_HALF:
        case QCU_PRECISION_BF16: return 2;
        default: return 0;
    }
}

inline bool prec_valid(int prec) { return prec_bytes(prec) != 0; }

// ---------------- storage traits ----------------
// S: scalar storage type; S2: complex storage pair; A: arithmetic type; A2 its pair.
template <typename S> struct St;
template <> struct St<double> {
    using S2 = double2;
    using A = double;
    using A2 = double2;
    __host__ __device__ static A2 ld(const S2& v) { return v; }
    __host__ __device__ static S2 cv(A2 v) { return v; }
};
template <> struct St<float> {
    using S2 = float2;
    using A = float;
    using A2 = float2;
    __host__ __device__ static A2 ld(const S2& v) { return v; }
    __host__ __device__ static S2 cv(A2 v) { return v; }
};
template <> struct St<__half> {
    using S2 = __half2;
    using A = float;
    using A2 = float2;
    __device__ static A2 ld(const S2& v) { return __half22float2(v); }
    __device__ static S2 cv(A2 v) { return __float22half2_rn(v); }
};
template <> struct St<__nv_bfloat16> {
    using S2 = __nv_bfloat162;
    using A = float;
    using A2 = float2;
    __device__ static A2 ld(const S2& v) { return __bfloat1622float2(v); }
    __device__ static S2 cv(A2 v) { return __float22bfloat162_rn(v); }
};

// conversion between any two storage pairs, via the wider arithmetic type
template <typename D, typename S>
__device__ __forceinline__ typename St<D>::S2 convert2(const typename St<S>::S2& v) {
    auto a = St<S>::ld(v);
    using DA2 = typename St<D>::A2;
    DA2 d;
    d.x = (typename St<D>::A)a.x;
    d.y = (typename St<D>::A)a.y;
    return St<D>::cv(d);
}

// ---------------- complex helpers ----------------
template <typename T> struct C2;
template <> struct C2<double> { using T2 = double2; };
template <> struct C2<float> { using T2 = float2; };

template <typename T2>
__host__ __device__ __forceinline__ T2 mk2(decltype(T2::x) a, decltype(T2::x) b) {
    T2 r;
    r.x = a;
    r.y = b;
    return r;
}

// acc += u * v
template <typename T2>
__device__ __forceinline__ void cmac(T2& acc, const T2& u, const T2& v) {
    acc.x = fma(u.x, v.x, acc.x);
    acc.x = fma(-u.y, v.y, acc.x);
    acc.y = fma(u.x, v.y, acc.y);
    acc.y = fma(u.y, v.x, acc.y);
}
// acc += conj(u) * v
template <typename T2>
__device__ __forceinline__ void cmac_conj(T2& acc, const T2& u, const T2& v) {
    acc.x = fma(u.x, v.x, acc.x);
    acc.x = fma(u.y, v.y, acc.x);
    acc.y = fma(u.x, v.y, acc.y);
    acc.y = fma(-u.y, v.x, acc.y);
}

// Dispatch on storage precision code.
template <typename F>
int dispatch_prec(int prec, F&& f) {
    switch (prec) {
        case QCU_PRECISION_DOUBLE: return f(double{});
        case QCU_PRECISION_SINGLE: return f(float{});
        case QCU_PRECISION_HALF: return f(__half{});
        case QCU_PRECISION_BF16: return f(__nv_bfloat16{});
        default: return set_error(QCU_ERR_INVALID, "unsupported precision code %d", prec);
    }
}

int sm_count();

// Resident blocks per SM of `kernel` at `block` threads (cached per kernel and size).
int blocks_per_sm(const void* kernel, int block, size_t smem = 0);

// Grid for a grid-stride kernel: enough blocks for the work, at most one full wave.
template <typename K>
static int resident_grid(K kernel, int block, int64_t work_items, size_t smem = 0) {
    const int per_sm = blocks_per_sm(reinterpret_cast<const void*>(kernel), block, smem);
    const int64_t want = (work_items + block - 1) / block;
    const int64_t cap = (int64_t)per_sm * sm_count();
    return (int)(want < cap ? (want < 1 ? 1 : want) : cap);
}

}  // namespace qcub
