// runtime.cu -- error state, device properties, occupancy cache, reduction scratch,
// hop dispatch.
#include <cstdarg>
#include <map>
#include <mutex>
#include <utility>

#include "dslash.h"
#include "workspace.h"

namespace qcub {

// ---------------- error state ----------------
static thread_local int g_status = QCU_SUCCESS;
static thread_local char g_message[512] = "";

int set_error(int status, const char* fmt, ...) {
    g_status = status;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_message, sizeof(g_message), fmt, ap);
    va_end(ap);
    return status;
}

void clear_error() {
    g_status = QCU_SUCCESS;
    g_message[0] = '\0';
}

int last_status() { return g_status; }
const char* last_message() { return g_message; }

// ---------------- device properties ----------------
static std::mutex g_mu;

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (cached[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1)
            n = 1;
        cached[dev] = n;
    }
    return cached[dev];
}

int blocks_per_sm(const void* kernel, int block, size_t smem) {
    static std::map<std::pair<const void*, int>, int> cache;
    std::lock_guard<std::mutex> lk(g_mu);
    auto key = std::make_pair(kernel, block * 65536 + (int)(smem / 16));
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem) != cudaSuccess ||
        per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    cache[key] = per_sm;
    return per_sm;
}

// ---------------- scratch ----------------
int scratch_alloc(Scratch* s) {
    s->max_blocks = kScratchBlocks;
    const size_t pbytes = sizeof(double2) * (size_t)kScratchBlocks * kMaxRedVals * kMaxRhs;
    QCUB_CUDA_CHECK(cudaMalloc(&s->partials, pbytes));
    QCUB_CUDA_CHECK(cudaMalloc(&s->counter, 256));
    QCUB_CUDA_CHECK(cudaMemset(s->counter, 0, 256));
    QCUB_CUDA_CHECK(cudaMalloc(&s->result, sizeof(double2) * kMaxRedVals * kMaxRhs));
    return QCU_SUCCESS;
}

void scratch_free(Scratch* s) {
    if (s->partials) cudaFree(s->partials);
    if (s->counter) cudaFree(s->counter);
    if (s->result) cudaFree(s->result);
    *s = Scratch{};
}

int device_scratch(const Scratch** out) {
    static Scratch per_dev[64];
    int dev = 0;
    QCUB_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_error(QCU_ERR_INVALID, "device index %d", dev);
    std::lock_guard<std::mutex> lk(g_mu);
    if (per_dev[dev].partials == nullptr) {
        int rc = scratch_alloc(&per_dev[dev]);
        if (rc) return rc;
    }
    *out = &per_dev[dev];
    return QCU_SUCCESS;
}

// ---------------- device error flag (bounded waits that gave up) ----------------
int* device_error_flag() {
    static int* per_dev[64] = {nullptr};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    if (per_dev[dev] == nullptr) {
        int* p = nullptr;
        if (cudaMalloc(&p, sizeof(int)) != cudaSuccess) return nullptr;
        cudaMemset(p, 0, sizeof(int));
        per_dev[dev] = p;
    }
    return per_dev[dev];
}

// ---------------- hop kernel selection ----------------
static int g_hop_kind = QCU_HOP_AUTO;

int hop_kind() { return g_hop_kind; }
void set_hop_kind(int k) { g_hop_kind = k; }

bool hop_tc_supported(int nc, int m, int prec);

// Kernel used when the selection is AUTO: the tuned choice for (n_color, m, precision)
// if one was recorded (qcuTuneHop / the tuning cache), else a static rule: the packed
// 16-bit kernel for FP16/BF16 storage where it applies, per-(site, RHS) SIMT otherwise.
int auto_hop_kind(int nc, int m, int prec);
int hop_tc_launch(const HopParams& p, int nc, int prec, bool dagger, int epi, cudaStream_t st);
bool hop16_supported(int nc, int m, int prec);
bool hop16_pairs_supported(int nc, int m, int prec);
int hop16_pairs_launch(const HopParams& p, int nc, int prec, bool dagger, int epi, cudaStream_t st);
bool hop_mma16_supported(int nc, int m, int prec);
int hop_mma16_launch(const HopParams& p, int nc, int prec, bool dagger, int epi, cudaStream_t st);
bool hop_mmal_supported(int nc, int m, int prec);
int hop_mmal_launch(const HopParams& p, int nc, int prec, bool dagger, int epi, bool staged, cudaStream_t st);
int hop16_launch(const HopParams& p, int nc, int prec, bool dagger, int epi, bool acc16, bool staged,
                 cudaStream_t st);

// ---------------- hop dispatch ----------------
template <typename S>
static int hop_nc(const HopParams& p, int nc, bool dagger, int epi, cudaStream_t st, bool cs) {
    switch (nc) {
        case 2: return launch_hop<2, S>(p, dagger, epi, st, cs);
        case 3: return launch_hop<3, S>(p, dagger, epi, st, cs);
        case 4: return launch_hop<4, S>(p, dagger, epi, st, cs);
        case 5: return launch_hop<5, S>(p, dagger, epi, st, cs);
        case 6: return launch_hop<6, S>(p, dagger, epi, st, cs);
        case 7: return launch_hop<7, S>(p, dagger, epi, st, cs);
        case 8: return launch_hop<8, S>(p, dagger, epi, st, cs);
        default: return set_error(QCU_ERR_UNSUPPORTED, "n_color=%d (supported: 2..8)", nc);
    }
}

bool hop_reads_tables(int nc, int m, int prec) {
    if (prec != QCU_PRECISION_HALF && prec != QCU_PRECISION_BF16) return false;
    int kind = g_hop_kind;
    if (kind == QCU_HOP_AUTO) kind = auto_hop_kind(nc, m, prec);
    return (kind == QCU_HOP_MMA_LINK || kind == QCU_HOP_MMA_LINK_DIRECT) && hop_mmal_supported(nc, m, prec);
}

int hop_launch(const HopParams& p, int nc, int prec, bool dagger, int epi, cudaStream_t st) {
    if (p.m < 1 || p.m > kMaxRhs) return set_error(QCU_ERR_INVALID, "m_rhs=%d outside [1, %d]", p.m, kMaxRhs);
    if (p.g.L[0] % 2 || p.g.L[0] < 2 || p.g.L[1] < 1 || p.g.L[2] < 1 || p.g.L[3] < 1)
        return set_error(QCU_ERR_INVALID, "lattice %dx%dx%dx%d (Lx must be even)", p.g.L[0], p.g.L[1],
                         p.g.L[2], p.g.L[3]);
    if (p.blocked) return hop16_pairs_launch(p, nc, prec, dagger, epi, st);
    int kind = g_hop_kind;
    if (kind == QCU_HOP_AUTO) kind = auto_hop_kind(nc, p.m, prec);
    if (kind == QCU_HOP_TENSOR && hop_tc_supported(nc, p.m, prec) &&
        reinterpret_cast<uintptr_t>(p.in) % 16 == 0)
        return hop_tc_launch(p, nc, prec, dagger, epi, st);
    if (kind == QCU_HOP_MMA16 && hop_mma16_supported(nc, p.m, prec))
        return hop_mma16_launch(p, nc, prec, dagger, epi, st);
    if ((kind == QCU_HOP_MMA_LINK || kind == QCU_HOP_MMA_LINK_DIRECT) && hop_mmal_supported(nc, p.m, prec))
        return hop_mmal_launch(p, nc, prec, dagger, epi, kind == QCU_HOP_MMA_LINK, st);
    if (kind == QCU_HOP_PACKED16_PAIRS && hop16_pairs_supported(nc, p.m, prec))
        return hop16_pairs_launch(p, nc, prec, dagger, epi, st);
    if ((kind == QCU_HOP_PACKED16 || kind == QCU_HOP_PACKED16_ACC16 || kind == QCU_HOP_PACKED16_STAGED ||
         kind == QCU_HOP_PACKED16_PAIRS) &&
        hop16_supported(nc, p.m, prec))
        return hop16_launch(p, nc, prec, dagger, epi, kind == QCU_HOP_PACKED16_ACC16,
                            kind == QCU_HOP_PACKED16_STAGED, st);
    const bool cs = (kind == QCU_HOP_SIMT_CS) && nc * p.m <= kRedThreads;
    return dispatch_prec(prec, [&](auto tag) { return hop_nc<decltype(tag)>(p, nc, dagger, epi, st, cs); });
}

}  // namespace qcub
