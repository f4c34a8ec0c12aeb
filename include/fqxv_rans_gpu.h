/*
 * fqxv_rans_gpu.h -- C ABI of the B200 (sm_100a) rANS Nx16 coder.
 *
 * A drop-in for the public API of the reference crate `fqxv-rans`
 * (crates/fqxv-rans/src/lib.rs) and its byte format (scalar.rs:8-20):
 * 32 interleaved states, 16-bit renormalisation, 12-bit frequency total,
 * order-0 and order-1 models. Every stream written here is byte-identical to
 * the reference encoder's on the same input and order, and every stream the
 * reference writes decodes here to the same bytes.
 *
 * Plain pointers and sizes only. Functions return an fqxv_rans_status; the
 * Malformed variants map 1:1 onto the reference's Error::Malformed messages
 * (fqxv_rans_status_message returns the reference's text).
 *
 * Threading: the single-call functions are re-entrant (they serialise on a
 * per-device default context). A fqxv_rans_ctx owns one CUDA stream and its
 * device arenas; calls on one context must not overlap, calls on different
 * contexts may.
 */
#ifndef FQXV_RANS_GPU_H
#define FQXV_RANS_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ----------------------------------------------------- */
typedef enum fqxv_rans_status {
    FQXV_RANS_OK = 0,
    /* Error::Malformed("truncated stream")                      scalar.rs:261 */
    FQXV_RANS_E_TRUNCATED = 1,
    /* Error::Malformed("unknown order tag")                     scalar.rs:153 */
    FQXV_RANS_E_UNKNOWN_ORDER = 2,
    /* Error::Malformed("rANS freq table exceeds TOTFREQ")       model.rs:165 */
    FQXV_RANS_E_FREQ_EXCEEDS = 3,
    /* Error::Malformed("rANS freq table does not sum to TOTFREQ") model.rs:169 */
    FQXV_RANS_E_FREQ_SUM = 4,
    /* Error::Malformed("symbol references absent context")      scalar.rs:206 */
    FQXV_RANS_E_ABSENT_CONTEXT = 5,
    /* Error::Malformed("rANS output length too large to allocate") model.rs:202;
     * here: the declared length exceeds the caller's output capacity. */
    FQXV_RANS_E_ALLOC = 6,
    /* Error::Malformed("rANS output length exceeds caller bound") lib.rs:228 */
    FQXV_RANS_E_BOUND = 7,
    /* Error::Malformed("truncated renorm stream") avx2.rs:207 -- only the
     * reference's SIMD backends say this; this decoder follows scalar.rs and
     * reports FQXV_RANS_E_TRUNCATED instead. Kept for numbering parity. */
    FQXV_RANS_E_TRUNCATED_RENORM = 8,
    /* Extended format only (fqxv_rans_x_gpu.h; no reference counterpart):
     * its transform data does not fit together. */
    FQXV_RANS_E_X_MALFORMED = 9,
    /* API errors (no reference counterpart). */
    FQXV_RANS_E_INVALID_ARG = 16,
    FQXV_RANS_E_DST_TOO_SMALL = 17,
    FQXV_RANS_E_CUDA = 18,
    FQXV_RANS_E_NO_DEVICE = 19,
    FQXV_RANS_E_OUT_OF_MEMORY = 20,
    FQXV_RANS_E_TIMEOUT = 21,
    FQXV_RANS_E_TOO_LARGE = 22
} fqxv_rans_status;

/* Order::Zero / Order::One (lib.rs:59-64), plus the two "encode both, keep the
 * smaller" selection rules the reference's callers apply:
 *   BEST_TIE0: ties keep order-0 -- fqxv-tokenizer/src/lib.rs:91-95 and
 *              fqxv/src/container/reorder.rs:597-609 (the permutation planes).
 *   BEST_TIE1: ties keep order-1 -- fqxv-lroverlap/src/codec.rs:293-306. */
enum {
    FQXV_RANS_ORDER0 = 0,
    FQXV_RANS_ORDER1 = 1,
    FQXV_RANS_BEST_TIE0 = 2,
    FQXV_RANS_BEST_TIE1 = 3
};

/* Backend (lib.rs:68-77). The GPU path ignores it: like the reference's
 * decode_with, every backend produces the same bytes. */
enum {
    FQXV_RANS_BACKEND_SCALAR = 0,
    FQXV_RANS_BACKEND_SSE42 = 1,
    FQXV_RANS_BACKEND_AVX2 = 2,
    FQXV_RANS_BACKEND_AVX512 = 3
};

/* The reference's message text for a status (static storage). */
const char *fqxv_rans_status_message(int status);

/* Library version string. */
const char *fqxv_rans_version(void);

/* ---- single-call API over host buffers (lib.rs) ---------------------------
 * Each call copies its input to the GPU, codes it there and copies the
 * result back. Rust's `Vec` return becomes a caller buffer of capacity `cap`
 * plus the produced length. */

/* Worst-case encoded length of an n-byte input: 9 + 2n + 640 (order 0) or
 * 9 + 2n + 131232 (order 1); 9 for n == 0. BEST_* modes take the order-1
 * bound. No reference counterpart (Rust grows a Vec). */
size_t fqxv_rans_encode_bound(size_t n, int order);

/* Replaces `pub fn encode(src: &[u8], order: Order) -> Result<Vec<u8>>`
 * (lib.rs:111). `order` may also be a BEST_* mode. */
int fqxv_rans_encode(const uint8_t *src, size_t n, int order, uint8_t *dst, size_t cap,
                     size_t *out_len);

/* Replaces `fn peek_output_len(src: &[u8]) -> Option<u64>` (lib.rs:207):
 * FQXV_RANS_E_TRUNCATED when src is shorter than 9 bytes. */
int fqxv_rans_peek_output_len(const uint8_t *src, size_t len, uint64_t *n);

/* Replaces `pub fn decode(src: &[u8]) -> Result<Vec<u8>>` (lib.rs:186).
 * A stream declaring more than `cap` bytes fails with FQXV_RANS_E_ALLOC at
 * the point the reference would allocate. */
int fqxv_rans_decode(const uint8_t *src, size_t len, uint8_t *dst, size_t cap, size_t *out_len);

/* Replaces `pub fn decode_bounded(src: &[u8], max_len: usize)` (lib.rs:226):
 * FQXV_RANS_E_BOUND when the header declares more than max_len, checked
 * before any decoding. */
int fqxv_rans_decode_bounded(const uint8_t *src, size_t len, size_t max_len, uint8_t *dst,
                             size_t cap, size_t *out_len);

/* Replaces `pub fn decode_with(src: &[u8], backend: Backend)` (lib.rs:241). */
int fqxv_rans_decode_with(const uint8_t *src, size_t len, int backend, uint8_t *dst, size_t cap,
                          size_t *out_len);

/* ---- contexts and the batched device API --------------------------------
 * No reference counterpart as one call: the reference codes independent
 * blocks on rayon workers (crates/fqxv/src/container/decompress.rs:46-52,
 * compress.rs:868); here a whole batch of blocks is one GPU pass. */

typedef struct fqxv_rans_ctx fqxv_rans_ctx;

/* One span of a device arena. */
typedef struct fqxv_rans_span {
    uint64_t offset;
    uint64_t length;
} fqxv_rans_span;

int fqxv_rans_ctx_create(int device, fqxv_rans_ctx **out);
void fqxv_rans_ctx_destroy(fqxv_rans_ctx *ctx);
/* The context's CUDA stream (a cudaStream_t). Work in a context is ordered
 * on this stream. */
void *fqxv_rans_ctx_stream(fqxv_rans_ctx *ctx);
/* Device bytes currently held by the context's arenas. */
uint64_t fqxv_rans_ctx_device_bytes(fqxv_rans_ctx *ctx);

/* Capacity the compacted output of encode_batch can need. */
uint64_t fqxv_rans_encode_batch_bound(const fqxv_rans_span *blocks, size_t nblocks, int order);

/* Encode `nblocks` blocks of device arena d_src (spans on the host) with one
 * order mode. The streams are written back to back into d_dst (device,
 * capacity dst_cap) in block order; out_spans[i] (host) receives stream i's
 * place and out_orders[i] (host, may be NULL) the order chosen. Synchronous.
 * `persistent` != 0 runs each stage as one launch over the whole batch (the
 * batched form); 0 launches every block separately (the plain per-block
 * form, for comparison). */
int fqxv_rans_encode_batch(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *blocks,
                           size_t nblocks, int order, uint8_t *d_dst, uint64_t dst_cap,
                           fqxv_rans_span *out_spans, int32_t *out_orders, int persistent);

/* Decode `nblocks` streams of d_src (spans on the host) into d_dst at the
 * caller's out_spans (offset, capacity). max_len applies decode_bounded's
 * check to every stream (UINT64_MAX: none). out_lens and status are host
 * arrays. Returns the first non-OK block status, or OK. Synchronous. */
int fqxv_rans_decode_batch(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *blocks,
                           size_t nblocks, uint64_t max_len, uint8_t *d_dst,
                           const fqxv_rans_span *out_spans, uint64_t *out_lens, int32_t *status,
                           int persistent);

/* Host-buffer batch forms of the two calls above: the input arena is copied
 * to the device, coded in one pass, and the results copied back (pinned host
 * memory makes the copies asynchronous DMA). For decode, a pinned (mapped)
 * destination of at least 4 MiB is instead written by the kernels in place
 * over the host link when the batch decodes slowly enough for the link
 * (estimated from the stream headers), overlapping the output transfer with
 * the decode; the destination bytes of a stream that fails are then
 * unspecified. Batches of 32 MiB or more run as up to four concurrent chunks
 * of consecutive blocks (the context's lock is held throughout), overlapping
 * one chunk's transfers with another's kernels.
 * out_spans/out_lens/status as above; for encode, out_spans index into
 * h_dst. */
int fqxv_rans_encode_batch_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, const fqxv_rans_span *blocks,
                                size_t nblocks, int order, uint8_t *h_dst, uint64_t dst_cap,
                                fqxv_rans_span *out_spans, int32_t *out_orders);
int fqxv_rans_decode_batch_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, const fqxv_rans_span *blocks,
                                size_t nblocks, uint64_t max_len, uint8_t *h_dst,
                                const fqxv_rans_span *out_spans, uint64_t *out_lens, int32_t *status);

/* ---- serving: continuous batching -----------------------------------------
 * No reference counterpart. A server owns n_workers contexts (CUDA streams)
 * on one device. Requests (one stream each) are admitted in arrival order
 * while their device-memory estimate fits under hbm_cap (0: 40 GiB); a free
 * worker takes every admitted request with the oldest request's kind, order
 * mode and size class (input sizes within a factor of four) and codes them as
 * one batched pass, so requests arriving while others run join the next pass
 * and passes of different workers overlap on the device. Workers are warmed
 * (pinned staging, one small pass per kernel path) before create returns.
 * A decompress request whose declared length exceeds its max_len completes
 * at submission with FQXV_RANS_E_BOUND. Results are byte-identical to the
 * single calls. */
typedef struct fqxv_rans_server fqxv_rans_server;

int fqxv_rans_server_create(int device, int n_workers, uint64_t hbm_cap, fqxv_rans_server **out);
/* Finishes queued work, then frees the server. */
void fqxv_rans_server_destroy(fqxv_rans_server *server);
/* kind 0: compress `src` with order mode `order`; kind 1: decompress `src`
 * with decode_bounded's `max_len`. The bytes are copied; *id identifies the
 * request. FQXV_RANS_E_TOO_LARGE when one request alone exceeds the cap. */
int fqxv_rans_server_submit(fqxv_rans_server *server, int kind, const uint8_t *src, size_t len, int order,
                            uint64_t max_len, uint64_t *id);
/* Wait up to timeout_ms (-1: no limit) for request id. On completion returns
 * FQXV_RANS_OK with its output length, its coding status and its latency
 * (submit to completion, microseconds); FQXV_RANS_E_TIMEOUT if not done. */
int fqxv_rans_server_wait(fqxv_rans_server *server, uint64_t id, int timeout_ms, size_t *out_len, int32_t *status,
                          double *latency_us);
/* Copy a completed request's output (cap >= its length) and release it. */
int fqxv_rans_server_take(fqxv_rans_server *server, uint64_t id, uint8_t *dst, size_t cap);
int fqxv_rans_server_stats(fqxv_rans_server *server, uint64_t *completed, uint64_t *batches,
                           uint64_t *peak_bytes, uint64_t *pending);

/* No counterpart in the reference. Encode one block that is already in device
 * memory without allocating any device memory, for callers that cannot call
 * cudaMalloc (a fixed device-memory budget reserved at start-up, an allocator
 * that must not be re-entered, a process that forbids driver allocations once
 * running). Its working memory is one file-scope device array of about 4.8 MiB
 * that every GPU loading the library holds until exit. d_src holds n <= 1 MiB
 * bytes (larger: FQXV_RANS_E_TOO_LARGE); the stream is written to d_dst, which
 * must hold fqxv_rans_encode_bound(n, order) bytes; its length goes to
 * *out_len. Work is queued on `stream` (a cudaStream_t, 0 = legacy default) and
 * the call returns once it is done. All calls share the array: calls whose
 * work overlaps on the GPU race and corrupt each other. Every call looks up
 * the array's address on the current device (so it stays valid across a
 * cudaDeviceReset); the first call on a device may load the library's device
 * code while doing so, so make it before any stream capture. */
int fqxv_rans_encode_noalloc(const uint8_t *d_src, size_t n, int order, uint8_t *d_dst, size_t dst_cap,
                             size_t *out_len, void *stream);

/* ---- launch shapes -------------------------------------------------------
 * No reference counterpart beyond Backend::detect (lib.rs:80-97). Every
 * context has integer launch-shape parameters: the decoder choice for wide
 * order-1 alphabets by stream count, the launch groups of the order-1
 * streams that bound a batch, CTAs per SM of each decode class, dense-table
 * group edges, the encode grid, the order-1 key array and the host-buffer
 * pipeline. They start from the tuning table of the device when one is found
 * (FQXV_RANS_TUNING, else tuning/<device>.json beside the package directory
 * of the library), else from the built-in rules. Names:
 *   o1_four_max_streams, o1_top_latency_pct, o1_top_max, o1_top_exclusive,
 *   o1_top_small_per_sm,
 *   cta_cap_o0, cta_cap_o1_small, cta_cap_o1_wide, cta_cap_o1_four,
 *   cta_cap_o1_global, cta_cap_o1_small_topped, cta_cap_o1_wide_topped,
 *   dense_edge_small, dense_edge_large,
 *   enc_run_ctas_per_sm, enc_run_ctas_per_sm_uniform, enc_o1_keys,
 *   host_enc_chunks, host_dec_chunks, host_in_place, host_out_mirror.
 * Unknown names and out-of-range values: FQXV_RANS_E_INVALID_ARG. Output
 * bytes never depend on them. */
int fqxv_rans_ctx_set_param(fqxv_rans_ctx *ctx, const char *name, int64_t value);
int fqxv_rans_ctx_get_param(fqxv_rans_ctx *ctx, const char *name, int64_t *value);
/* Path of the tuning table the context applied ("" when none). */
const char *fqxv_rans_ctx_tuning_source(fqxv_rans_ctx *ctx);

/* ---- per-stage device timing -------------------------------------------
 * When enabled, every kernel launch of a context is bracketed by CUDA events
 * on the context's stream and its duration accumulated per stage. Launch
 * counts are kept whether or not timing is on. Launches of one stage may run
 * side by side on several CUDA streams (the decode groups of a batch), so
 * `ms` (the sum of launch durations) can exceed the time the stage took;
 * `wall_ms` is that time: per call, from the stage's first launch start to
 * its last launch end, summed over calls. */
typedef struct fqxv_rans_stage_stat {
    char name[24];
    uint64_t launches;
    double ms;
    uint64_t bytes;   /* algorithmic bytes (input read + output written) of those launches */
    double wall_ms;       /* first launch start to last launch end, per call, summed */
    uint32_t ctas_per_sm; /* decode stages: CTAs per SM of the largest launch shape */
    uint32_t smem_bytes;  /* decode stages: dynamic shared memory per CTA, largest */
} fqxv_rans_stage_stat;

int fqxv_rans_ctx_set_profiling(fqxv_rans_ctx *ctx, int on);
/* Copies up to `cap` stage records into `out`, the count into *n; reset != 0
 * clears the counters afterwards. */
int fqxv_rans_ctx_stage_stats(fqxv_rans_ctx *ctx, fqxv_rans_stage_stat *out, int cap, int *n, int reset);

#ifdef __cplusplus
}
#endif
#endif
