// fqxv_rans_encode_noalloc: encode one device-resident block without
// allocating any device memory.
//
// The regular entry points grow per-context device arenas with cudaMalloc.
// Some callers cannot allow that: code running under a fixed device-memory
// budget carved out up front, code inside a memory pool or allocator that
// must not be re-entered, or a host process that forbids driver allocations
// after start-up. For them this entry point keeps all of its working memory
// (block descriptor, encode tables, histogram and renorm-word scratch) in one
// file-scope __device__ array of kNoAllocScratchBytes, reserved on every GPU
// that loads the library until the process exits. The caller passes the
// input and output device buffers.
//
// The largest input one call accepts is kNoAllocMaxBytes (1 MiB); larger
// inputs are rejected with FQXV_RANS_E_TOO_LARGE.
//
// Every call shares the one array and it keeps whatever the previous call
// left there; the kernels clear what must start at zero. Two calls whose work
// overlaps on the GPU (different streams, or different host threads without
// ordering) race on the array and corrupt each other's output.
//
// Every call looks up the array's device address on the current device
// (cudaGetSymbolAddress), so the address stays right after a
// cudaDeviceReset reloads the module. The first call on a device may load
// the module while doing so; make that first call before any stream capture.
#include "rans_internal.cuh"

namespace fqxv {

namespace {

constexpr uint64_t kNoAllocMaxBytes = 1ull << 20;
constexpr uint64_t kOffBlock = 0;
constexpr uint64_t kOffOrder = 1024;
constexpr uint64_t kOffJobs = 1280;
constexpr uint64_t kOffQueue = 2048;
constexpr uint64_t kOffTotal = 2064;
constexpr uint64_t kOffTbl = 4096;
constexpr uint64_t kTblBytes = 528384;  // >= enc_table_bytes(n) for every n
constexpr uint64_t kOffHist = kOffTbl + kTblBytes;
constexpr uint64_t kHistBytes = 65536 * 4;
constexpr uint64_t kOffWords = kOffHist + kHistBytes;
constexpr uint64_t kWordsBytes = 2 * kNoAllocMaxBytes * 2;  // two orders x n x u16
constexpr uint64_t kNoAllocScratchBytes = kOffWords + kWordsBytes;
static_assert(sizeof(EncBlock) <= kOffOrder, "descriptor region too small");

}  // namespace

static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

// Fills the descriptor, the one-entry block order, the job list and the queue
// counter for a single block of n bytes coded in `mode`.
__global__ void noalloc_setup_kernel(uint64_t n, int mode) {
    if (threadIdx.x != 0) return;
    uint8_t *s = g_noalloc_scratch;
    EncBlock *B = reinterpret_cast<EncBlock *>(s + kOffBlock);
    uint8_t *raw = reinterpret_cast<uint8_t *>(B);
    for (unsigned i = 0; i < sizeof(EncBlock); i++) raw[i] = 0;
    B->src_off = 0;
    B->n = n;
    B->mode = mode;
    B->word_off[0] = 0;
    B->word_off[1] = n;
    B->tbl_off = 0;
    *reinterpret_cast<uint32_t *>(s + kOffOrder) = 0;
    EncJob *J = reinterpret_cast<EncJob *>(s + kOffJobs);
    int nj = 0;
    if (mode != FQXV_RANS_ORDER0) J[nj++] = EncJob{0, 1};
    if (mode != FQXV_RANS_ORDER1) J[nj++] = EncJob{0, 0};
    *reinterpret_cast<int *>(s + kOffQueue) = 0;
    *reinterpret_cast<uint64_t *>(s + kOffTotal) = 0;
}

}  // namespace fqxv

using namespace fqxv;

namespace {

// Device address of the scratch array on the current device. The lookup is
// repeated on every call: a cached address would go stale when
// cudaDeviceReset unloads the module and a later call loads it again.
int noalloc_scratch(uint8_t **out) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return FQXV_RANS_E_CUDA;
    }
    *out = static_cast<uint8_t *>(p);
    return FQXV_RANS_OK;
}

}  // namespace

extern "C" int fqxv_rans_encode_noalloc(const uint8_t *d_src, size_t n, int order, uint8_t *d_dst,
                                        size_t dst_cap, size_t *out_len, void *stream) {
    if (!out_len || !d_dst || (n && !d_src)) return FQXV_RANS_E_INVALID_ARG;
    if (order < FQXV_RANS_ORDER0 || order > FQXV_RANS_BEST_TIE1) return FQXV_RANS_E_INVALID_ARG;
    if (n > kNoAllocMaxBytes) return FQXV_RANS_E_TOO_LARGE;
    if (dst_cap < fqxv_rans_encode_bound(n, order)) return FQXV_RANS_E_DST_TOO_SMALL;
    int dev = 0;  // a current device must exist
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return FQXV_RANS_E_NO_DEVICE;
    }
    uint8_t *s = nullptr;
    const int st = noalloc_scratch(&s);
    if (st != FQXV_RANS_OK) return st;
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    EncBlock *B = reinterpret_cast<EncBlock *>(s + kOffBlock);
    const uint32_t *ord = reinterpret_cast<const uint32_t *>(s + kOffOrder);
    const EncJob *jobs = reinterpret_cast<const EncJob *>(s + kOffJobs);
    int *queue = reinterpret_cast<int *>(s + kOffQueue);
    uint64_t *total = reinterpret_cast<uint64_t *>(s + kOffTotal);
    uint8_t *tbl = s + kOffTbl;
    uint32_t *hist = reinterpret_cast<uint32_t *>(s + kOffHist);
    uint16_t *words = reinterpret_cast<uint16_t *>(s + kOffWords);
    const int njobs = (order == FQXV_RANS_BEST_TIE0 || order == FQXV_RANS_BEST_TIE1) ? 2 : 1;

    noalloc_setup_kernel<<<1, 32, 0, cs>>>(n, order);
    if (launch_enc_model(d_src, B, ord, 1, tbl, hist, nullptr, 1, kModelCluster, cs) != cudaSuccess) {
        cudaGetLastError();
        return FQXV_RANS_E_CUDA;
    }
    launch_enc_run(d_src, B, jobs, njobs, tbl, words, queue, nullptr, 1, cs);
    launch_enc_select_scan(B, 1, total, cs);
    launch_enc_pack(B, 1, tbl, words, d_dst, 1, cs);
    uint64_t len = 0;
    if (cudaGetLastError() != cudaSuccess) return FQXV_RANS_E_CUDA;
    if (cudaMemcpyAsync(&len, total, sizeof len, cudaMemcpyDeviceToHost, cs) != cudaSuccess ||
        cudaStreamSynchronize(cs) != cudaSuccess) {
        cudaGetLastError();
        return FQXV_RANS_E_CUDA;
    }
    *out_len = (size_t)len;
    return FQXV_RANS_OK;
}
