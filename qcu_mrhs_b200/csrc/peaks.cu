// peaks.cu -- arithmetic peak microbenchmarks: the compute ceilings the hop kernels are
// measured against (FP64 and FP32 fused multiply-add on the CUDA cores, FP64 warp MMA, and
// the 16-bit warp MMA with FP32 accumulation that the link-operand hop issues).
//
// Each thread (FMA kinds) or warp (MMA kinds) runs `iters` rounds of 8 independent
// operations, so the pipe sees 8 chains per thread and every resident warp; the launch is 4
// blocks of 256 threads per SM.  The rate is the FLOPs of the launch over its CUDA-event
// time on the caller's stream (one warm-up launch first).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"

namespace qcub {

namespace {

constexpr int kPThreads = 256;
constexpr int kPBlocksPerSm = 4;
constexpr int kPChains = 8;

template <typename T>
__global__ void __launch_bounds__(kPThreads) fma_peak_kernel(T* out, int iters, T a, T b) {
    T x[kPChains];
#pragma unroll
    for (int k = 0; k < kPChains; ++k) x[k] = (T)(threadIdx.x + k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kPChains; ++k) x[k] = fma(x[k], a, b);
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < kPChains; ++k) s += x[k];
    if (s == (T)-1) out[0] = s;   // keeps the chains live; never true for the inputs used
}

// FP64 warp MMA m8n8k4: D (8x8, 2 per lane) = A (8x4, 1 per lane) B (4x8, 1 per lane) + C
__global__ void __launch_bounds__(kPThreads) dmma_peak_kernel(double* out, int iters, double a, double b) {
    double d[kPChains][2];
#pragma unroll
    for (int k = 0; k < kPChains; ++k) d[k][0] = d[k][1] = 0.0;
    const double av = a + threadIdx.x * 1e-9, bv = b;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kPChains; ++k)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                         : "+d"(d[k][0]), "+d"(d[k][1])
                         : "d"(av), "d"(bv));
    }
    double s = 0;
#pragma unroll
    for (int k = 0; k < kPChains; ++k) s += d[k][0] + d[k][1];
    if (s == -1.0) out[0] = s;
}

// 16-bit warp MMA m16n8k16 with FP32 accumulation (BF = bf16 operands, else fp16)
template <bool BF>
__global__ void __launch_bounds__(kPThreads) hmma_peak_kernel(double* out, int iters, uint32_t a, uint32_t b) {
    float d[kPChains][4];
#pragma unroll
    for (int k = 0; k < kPChains; ++k) d[k][0] = d[k][1] = d[k][2] = d[k][3] = 0.f;
    const uint32_t av = a ^ (threadIdx.x & 1u);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kPChains; ++k) {
            if (BF)
                asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%4,%4,%4}, "
                             "{%5,%5}, {%0,%1,%2,%3};"
                             : "+f"(d[k][0]), "+f"(d[k][1]), "+f"(d[k][2]), "+f"(d[k][3])
                             : "r"(av), "r"(b));
            else
                asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%4,%4,%4}, "
                             "{%5,%5}, {%0,%1,%2,%3};"
                             : "+f"(d[k][0]), "+f"(d[k][1]), "+f"(d[k][2]), "+f"(d[k][3])
                             : "r"(av), "r"(b));
        }
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < kPChains; ++k) s += d[k][0] + d[k][1] + d[k][2] + d[k][3];
    if (s == -1.f) out[0] = s;
}

}  // namespace

}  // namespace qcub

extern "C" int qcuPeakRate(int kind, int iters, double* flops, void* stream) {
    using namespace qcub;
    if (!flops || iters < 1) return set_error(QCU_ERR_INVALID, "qcuPeakRate: flops pointer and iters >= 1 required");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int blocks = kPBlocksPerSm * sm_count();
    const double warps = (double)blocks * (kPThreads / 32);
    const double threads = (double)blocks * kPThreads;
    double per_round = 0.0;   // FLOPs of one round of the launch
    switch (kind) {
        case QCU_PEAK_DFMA:
        case QCU_PEAK_FFMA: per_round = threads * kPChains * 2.0; break;
        case QCU_PEAK_DMMA: per_round = warps * kPChains * 2.0 * 8 * 8 * 4; break;
        case QCU_PEAK_HMMA:
        case QCU_PEAK_BMMA: per_round = warps * kPChains * 2.0 * 16 * 8 * 16; break;
        default: return set_error(QCU_ERR_INVALID, "qcuPeakRate: kind %d", kind);
    }
    double* sink = nullptr;
    QCUB_CUDA_CHECK(cudaMallocAsync(&sink, sizeof(double), st));
    auto launch = [&]() {
        switch (kind) {
            case QCU_PEAK_DFMA:
                fma_peak_kernel<double><<<blocks, kPThreads, 0, st>>>(sink, iters, 0.999999, 1e-7);
                break;
            case QCU_PEAK_FFMA:
                fma_peak_kernel<float><<<blocks, kPThreads, 0, st>>>(reinterpret_cast<float*>(sink), iters, 0.999f,
                                                                     1e-4f);
                break;
            case QCU_PEAK_DMMA: dmma_peak_kernel<<<blocks, kPThreads, 0, st>>>(sink, iters, 1e-3, 1e-3); break;
            case QCU_PEAK_HMMA:   // fp16 pairs (1e-3, 1e-3) and (1e-2, 1e-2)
                hmma_peak_kernel<false><<<blocks, kPThreads, 0, st>>>(sink, iters, 0x141A141Au, 0x211F211Fu);
                break;
            default:              // bf16 pairs (1e-3, 1e-3) and (1e-2, 1e-2)
                hmma_peak_kernel<true><<<blocks, kPThreads, 0, st>>>(sink, iters, 0x3A833A83u, 0x3C243C24u);
                break;
        }
    };
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = QCU_SUCCESS;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        rc = set_error(QCU_ERR_CUDA, "qcuPeakRate: event creation failed");
    } else {
        launch();   // warm-up
        cudaEventRecord(e0, st);
        launch();
        cudaEventRecord(e1, st);
        const cudaError_t e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e != cudaSuccess || cudaGetLastError() != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess ||
            ms <= 0.f)
            rc = set_error(QCU_ERR_CUDA, "qcuPeakRate: launch failed: %s", cudaGetErrorString(e));
        else
            *flops = per_round * iters / (ms * 1e-3);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFreeAsync(sink, st);
    return rc;
}
