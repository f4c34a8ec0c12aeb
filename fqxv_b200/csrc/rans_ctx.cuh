// Device context shared by the C-ABI translation units (rans_capi.cu,
// frame_capi.cu): arenas, staging buffers, streams and stage timers of one
// fqxv_rans_ctx. Nothing here is part of the public ABI.
#pragma once

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "rans_internal.cuh"

namespace fqxv {

// Grow-only device buffer. Growth waits for the owning stream first, so a
// buffer is never freed under a kernel that still reads it.
struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t want, cudaStream_t s) {
        if (want <= cap) return cudaSuccess;
        size_t nc = std::max(want, cap + cap / 2);
        nc = align_up(nc, 1 << 20);
        if (p) {
            cudaStreamSynchronize(s);
            cudaFree(p);
            p = nullptr;
            cap = 0;
        }
        cudaError_t e = cudaMalloc(&p, nc);
        if (e != cudaSuccess) {
            cudaGetLastError();
            e = cudaMalloc(&p, want);
            if (e != cudaSuccess) {
                p = nullptr;
                return e;
            }
            nc = want;
        }
        cap = nc;
        return cudaSuccess;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    template <class T>
    T *as() const { return reinterpret_cast<T *>(p); }
};

struct HostBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t want) {
        if (want <= cap) return cudaSuccess;
        size_t nc = align_up(std::max(want, cap + cap / 2), 1 << 16);
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaHostAlloc(&p, nc, cudaHostAllocDefault);
        if (e != cudaSuccess) {
            p = nullptr;
            return e;
        }
        cap = nc;
        return cudaSuccess;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
};

// Decode launch groups: order-0; order-1 small alphabets; order-1 wide
// alphabets in three table-size ranges; the order-1 streams that bound the
// batch by their serial time, wide alphabets (four-warp decoder) and small
// ones, each group on SMs of its own; order-1 global tables.
constexpr int kGroupDense0 = 2;   // first of the three dense table-size groups
constexpr int kDenseGroups = 3;
constexpr int kGroupFourTop = kGroupDense0 + kDenseGroups;
constexpr int kGroupSmallTop = kGroupFourTop + 1;
constexpr int kGroups = kGroupSmallTop + 2;

enum Stage {
    kStEncModel, kStEncRun, kStEncScan, kStEncPack, kStDecParse, kStDecO0, kStDecO1Dense, kStDecO1Global,
    kStDecO1Small, kStDecO1Wide, kStCrcPlan, kStCrc, kStFrameCopy, kStFrameWalk, kStXEncode, kStXDecode, kStages
};
const char *const kStageNames[kStages] = {"enc_model", "enc_run", "enc_select_scan", "enc_pack",
                                          "dec_parse", "dec_o0", "dec_o1_dense", "dec_o1_global",
                                          "dec_o1_small", "dec_o1_wide", "crc_plan", "crc32c",
                                          "frame_copy_crc", "frame_walk", "x_encode", "x_decode"};

// Launch-shape parameters of a context (rans_tuning.cu): defaults are the
// library's run-time rules; a tuning table measured on the device replaces
// them.
struct Tuning {
    // Order-1 streams of more than kSmallMaxNd symbols with shared-memory
    // tables: a launch group of fewer than this many goes to the four-warp
    // decoder (one stream per SM), larger groups to the one-warp decoder
    // (several per SM). -1: the SM count.
    int64_t o1_four_max_streams = -1;
    // Order-1 streams whose serial decode alone outlasts o1_top_latency_pct %
    // of the batch's throughput-bound time -- the o1_top_max longest of them
    // -- form launch groups of their own (the batch lasts at least as long as
    // its longest serial chain): wide alphabets on the four-warp decoder,
    // small ones on the one-warp decoder. o1_top_max -1: half the SM count.
    int64_t o1_top_latency_pct = 75;
    int64_t o1_top_max = -1;
    // 1: those two groups run one CTA per SM with no other CTA beside it
    // (their CTAs claim the SM's shared memory), so their serial chains are
    // not slowed by the rest of the batch; 0: they share.
    int64_t o1_top_exclusive = 1;
    // CTAs per SM of the small-alphabet top group when exclusive: each is one
    // warp, so up to four can hold an SM together, one per scheduler.
    int64_t o1_top_small_per_sm = 4;
    // CTAs per SM of each decode class, at most (the occupancy API bounds it too)
    int64_t cta_cap_o0 = 32, cta_cap_o1_small = 32, cta_cap_o1_wide = 32, cta_cap_o1_four = 8,
            cta_cap_o1_global = 32;
    // the same for the one-warp classes outside the top groups when a batch
    // has top groups
    int64_t cta_cap_o1_small_topped = 4, cta_cap_o1_wide_topped = 3;
    // table-image sizes cutting the other dense wide-alphabet streams into
    // launch groups (a launch's shared memory is its largest member's)
    int64_t dense_edge_small = 40 << 10, dense_edge_large = 80 << 10;
    // encode kernel grid, CTAs per SM
    int64_t enc_run_ctas_per_sm = 2;
    // the same for batches of like-sized blocks (no block above four times
    // the mean)
    int64_t enc_run_ctas_per_sm_uniform = 3;
    // Order-1 encode: 1, the model kernel stores each position's table index
    // (u16) for the encode kernel to read back; 0, the encode kernel derives
    // it from the byte and its predecessor (no per-position array).
    int64_t enc_o1_keys = 1;
    // Host-buffer calls: chunks a batch of 32 MiB or more is cut into (one
    // sub-context and host thread each), for encode (the input copy of one
    // chunk overlaps the encode of the one before) and decode (a decode is
    // bound by its longest streams, and chunks decoded side by side slowed
    // config2's host decode from 74 to 123 ms); whether a decode reads its pinned
    // input in place (-1: when the batch is slow and has hundreds of
    // streams, 0: never, 1: whenever it is pinned); whether the decoding
    // CTAs copy each finished stream to a large pinned destination (1) or
    // the output is copied once the batch is done (0).
    int64_t host_enc_chunks = 4;
    int64_t host_dec_chunks = 1;
    int64_t host_in_place = -1;
    int64_t host_out_mirror = 1;
    std::string source;  // the table file applied (empty: defaults)
};
int tuning_set(Tuning &t, const char *key, int64_t value);
int tuning_get(const Tuning &t, const char *key, int64_t &value);
void tuning_load(Tuning &t, int device);

// CUDA-event brackets around each kernel launch on the context's stream.
// Durations are collected after the call's final synchronisation. Launches of
// one stage can run side by side on several streams (the decode groups), so
// besides the sum of launch durations (`ms`) the timer keeps each stage's
// wall time on the device (`wall_ms`): from its first launch's start to its
// last launch's end within a call, measured against an event recorded on the
// context's stream before the call's first launch (every later launch, on any
// of the context's streams, is ordered after it).
struct StageTimer {
    bool on = false;
    struct Pending {
        int stage;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;
    cudaEvent_t origin = nullptr;
    double ms[kStages] = {};
    double wall_ms[kStages] = {};
    uint64_t launches[kStages] = {};
    uint64_t bytes[kStages] = {};   // algorithmic bytes moved by the stage's launches
    // launch shape, largest over the stage's launches: CTAs per SM and
    // dynamic shared memory per CTA
    uint32_t ctas_per_sm[kStages] = {};
    uint32_t smem_bytes[kStages] = {};
    void shape(int stage, int per_sm, uint32_t smem) {
        ctas_per_sm[stage] = std::max(ctas_per_sm[stage], (uint32_t)std::max(per_sm, 0));
        smem_bytes[stage] = std::max(smem_bytes[stage], smem);
    }
    cudaEvent_t get() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        return e;
    }
    // Returns the start event (or null); pass it to end(). The first launch
    // of a call also records the call's origin on the same stream.
    cudaEvent_t begin(cudaStream_t s) {
        if (!on) return nullptr;
        if (!origin) {
            origin = get();
            if (origin) cudaEventRecord(origin, s);
        }
        cudaEvent_t a = get();
        if (a) cudaEventRecord(a, s);
        return a;
    }
    void end(int stage, cudaEvent_t a, cudaStream_t s) {
        launches[stage]++;
        if (!a) return;
        cudaEvent_t b = get();
        if (!b) return;
        cudaEventRecord(b, s);
        pending.push_back({stage, a, b});
    }
    void collect() {
        double lo[kStages], hi[kStages];
        for (int i = 0; i < kStages; i++) {
            lo[i] = 1e300;
            hi[i] = -1e300;
        }
        for (auto &p : pending) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, p.a, p.b) == cudaSuccess) ms[p.stage] += t;
            else cudaGetLastError();
            float ta = 0.f, tb = 0.f;
            if (origin && cudaEventElapsedTime(&ta, origin, p.a) == cudaSuccess &&
                cudaEventElapsedTime(&tb, origin, p.b) == cudaSuccess) {
                lo[p.stage] = std::min(lo[p.stage], (double)ta);
                hi[p.stage] = std::max(hi[p.stage], (double)tb);
            } else {
                cudaGetLastError();
            }
            pool.push_back(p.a);
            pool.push_back(p.b);
        }
        for (int i = 0; i < kStages; i++)
            if (hi[i] >= lo[i]) wall_ms[i] += hi[i] - lo[i];
        pending.clear();
        if (origin) pool.push_back(origin);
        origin = nullptr;
    }
    void release() {
        for (auto &p : pending) {
            pool.push_back(p.a);
            pool.push_back(p.b);
        }
        pending.clear();
        if (origin) pool.push_back(origin);
        origin = nullptr;
        for (auto e : pool) cudaEventDestroy(e);
        pool.clear();
    }
};


struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

// Device address of a pinned, mapped host buffer (nullptr for any other
// memory): with unified addressing a kernel can load and store it directly.
void *mapped_device_ptr(const void *h);

}  // namespace fqxv

namespace fqxv {
// Frees a context's extended-format arenas (rans_x.cu).
void x_release(fqxv_rans_ctx *ctx);
// fqxv_rans_encode_batch / fqxv_rans_decode_batch (persistent form) for
// callers that already hold ctx->mu and have the context's device current.
int encode_batch_locked(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *blocks, size_t nb, int mode,
                        uint8_t *d_dst, uint64_t dst_cap, fqxv_rans_span *out_spans, int32_t *out_orders);
int decode_batch_locked(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *blocks, size_t nb,
                        uint64_t max_len, uint8_t *d_dst, const fqxv_rans_span *out_spans, uint64_t *out_lens,
                        int32_t *status);
}  // namespace fqxv

struct fqxv_rans_ctx {
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    cudaStream_t aux[fqxv::kGroups] = {};   // decode launch groups run side by side
    cudaEvent_t ev_fork = nullptr, ev_join[fqxv::kGroups] = {};
    std::mutex mu;
    // encode
    fqxv::DevBuf e_blocks, e_order, e_jobs, e_tbl, e_words, e_hist, e_misc, e_keys;
    // decode
    fqxv::DevBuf d_streams, d_order, d_tbl, d_misc;
    // single-call staging
    fqxv::DevBuf io_in, io_out;
    // CRC-32C and block frames: targets, pieces, results
    fqxv::DevBuf f_targets, f_pieces, f_out;
    fqxv::HostBuf h_stage;
    fqxv::HostBuf h_io;
    fqxv::StageTimer timer;
    // Polls of a decode kernel's first wait for its table copy (a drain with
    // the full bound follows a wait that gives up). Only the test-only
    // setter in fqxv_rans_gpu_testing.h lowers it.
    uint32_t first_polls = fqxv::kWaitPolls;
    fqxv::Tuning tune;
    // arenas of the extended-format calls (rans_x.cu), created on first use
    // and freed by fqxv::x_release
    void *xb = nullptr;
    // host-buffer batches cut into chunks run one chunk per sub-context
    std::vector<fqxv_rans_ctx *> sub;
    template <class F>
    void for_each_buf(F &&f) {
        fqxv::DevBuf *all[] = {&e_blocks, &e_order, &e_jobs, &e_tbl, &e_words, &e_hist, &e_misc,
                               &e_keys, &d_streams, &d_order, &d_tbl, &d_misc, &io_in, &io_out,
                               &f_targets, &f_pieces, &f_out};
        for (auto *b : all) f(*b);
    }
    uint64_t device_bytes() {
        uint64_t t = 0;
        for_each_buf([&](fqxv::DevBuf &b) { t += b.cap; });
        for (auto *c : sub) t += c->device_bytes();
        return t;
    }
};

#define CK(x)                                                          \
    do {                                                               \
        cudaError_t e_ = (x);                                          \
        if (e_ != cudaSuccess) {                                       \
            cudaGetLastError();                                        \
            return e_ == cudaErrorMemoryAllocation ? FQXV_RANS_E_OUT_OF_MEMORY \
                                                   : FQXV_RANS_E_CUDA; \
        }                                                              \
    } while (0)
