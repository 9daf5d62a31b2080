// noalloc.cu -- qcuMrhsDotcNoAlloc: the multi-RHS inner product without any device
// allocation, for callers that cannot call cudaMalloc.
//
// qcuMrhsDotc keeps its per-block partial sums and its ticket counter in scratch
// memory that the library allocates with cudaMalloc on first use.  Some callers
// cannot allow that: an application whose device memory is entirely owned by another
// allocator (a framework's caching allocator, a pre-sized memory pool) or a caller on
// a code path where allocating is not permitted.  This variant keeps that scratch in
// a fixed file-scope device array instead.
//
// Limits and rules:
//   - scratch size is fixed at compile time: kNoAllocBlocks blocks x 64 RHS partial sums
//     (1 MiB) plus one 256-byte counter slot; every GPU that loads the library holds
//     this array until the process exits;
//   - m_rhs is limited to 64 (QCU_MAX_RHS); larger m is rejected with QCU_ERR_INVALID;
//     any vector length is accepted (the grid is capped at kNoAllocBlocks and strides);
//   - the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call before
//     any stream capture on the device;
//   - every call shares the one array: the counter is cleared (cudaMemsetAsync, no
//     allocation) at the start of each call, and calls whose kernels overlap on the
//     GPU (different streams, or different host threads) race on the array.
#include <mutex>

#include "blas_impl.cuh"

namespace qcub {

constexpr int kNoAllocBlocks = 1024;
constexpr size_t kNoAllocCounterBytes = 256;
constexpr size_t kNoAllocBytes =
    kNoAllocCounterBytes + sizeof(double2) * (size_t)kNoAllocBlocks * kMaxRhs;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[64] = {nullptr};
}  // namespace

// Device address of g_noalloc_scratch on the current device (looked up once per device).
static int noalloc_scratch(void** out) {
    int dev = 0;
    QCUB_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_error(QCU_ERR_INVALID, "device index %d", dev);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (g_noalloc_ptr[dev] == nullptr) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr)
            return set_error(QCU_ERR_CUDA, "cudaGetSymbolAddress(no-alloc scratch): %s", cudaGetErrorString(e));
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return QCU_SUCCESS;
}

template <typename S>
static int dotc_noalloc_t(double2* res, const void* a, const void* b, int64_t len, int m, void* scratch,
                          cudaStream_t st) {
    using S2 = typename St<S>::S2;
    unsigned char* base = static_cast<unsigned char*>(scratch);
    unsigned* counter = reinterpret_cast<unsigned*>(base);
    double2* partials = reinterpret_cast<double2*>(base + kNoAllocCounterBytes);
    QCUB_CUDA_CHECK(cudaMemsetAsync(counter, 0, sizeof(unsigned), st));
    const int block = rhs_block(m);
    auto k = dotc_kernel<S>;
    int grid = resident_grid(k, block, len * m);
    if (grid > kNoAllocBlocks) grid = kNoAllocBlocks;   // [grid][m] partials fit the array
    RedArgs ra{partials, counter, res, nullptr, nullptr, FIN_NONE};
    k<<<grid, block, 0, st>>>(static_cast<const S2*>(a), static_cast<const S2*>(b), len * m, m, ra);
    QCUB_CHECK_LAUNCH();
    return QCU_SUCCESS;
}

}  // namespace qcub

using namespace qcub;

extern "C" int qcuMrhsDotcNoAlloc(void* res, const void* a, const void* b, int64_t len, int m,
                                  int precision, void* stream) {
    clear_error();
    if (m < 1 || m > kMaxRhs)
        return set_error(QCU_ERR_INVALID, "qcuMrhsDotcNoAlloc: m_rhs=%d outside [1, %d] (fixed scratch size)", m,
                         kMaxRhs);
    if (len < 0) return set_error(QCU_ERR_INVALID, "qcuMrhsDotcNoAlloc: negative vector length");
    if (!res || !a || !b) return set_error(QCU_ERR_INVALID, "qcuMrhsDotcNoAlloc: null pointer");
    void* scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    return dispatch_prec(precision, [&](auto tag) {
        return dotc_noalloc_t<decltype(tag)>(static_cast<double2*>(res), a, b, len, m, scratch,
                                            static_cast<cudaStream_t>(stream));
    });
}
