// Internal definitions shared by the encode, decode and C-ABI translation
// units of libfqxv_rans_gpu.so. Nothing here is part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/fqxv_rans_gpu.h"

namespace fqxv {

// crates/fqxv-rans/src/model.rs:9-19
constexpr uint32_t kScaleBits = 12;
constexpr uint32_t kTotFreq = 1u << kScaleBits;
constexpr uint32_t kRansL = 1u << 16;
constexpr int kStates = 32;

// scalar.rs:8-20: [u8 order][u64 n] ++ tables ++ [32 x u32 states] ++ words
constexpr uint64_t kHdr = 9;
constexpr uint64_t kO0Tables = 512;         // 256 x u16
constexpr uint64_t kO1Bitmap = 32;          // context presence bitmap
constexpr uint64_t kO1Table = 512;          // 256 x u16 per present context
constexpr uint64_t kStatesBytes = 4 * kStates;

// Persistent-kernel shapes.
constexpr int kModelThreads = 512;          // model kernel: threads per CTA
constexpr int kModelCluster = 8;            // model kernel: CTAs (one cluster) per large block
constexpr uint64_t kModelClusterMin = 256 << 10;  // smaller blocks get one CTA each
constexpr int kEncWarpsPerCta = 4;          // encode: one warp per (block, order)
constexpr int kDecWarpsPerCta = 4;          // decode: one warp per stream
constexpr int kParseThreads = 256;          // decode header/table kernel
constexpr int kPackThreads = 256;           // output compaction
constexpr int kPackParts = 8;               // output compaction: CTAs per block

// Encode-side descriptor of one input block (device resident).
struct EncBlock {
    uint64_t src_off;       // offset of the block in the input arena
    uint64_t n;             // block length in bytes
    uint64_t word_off[2];   // word-scratch region (u16 units) per order; n words each
    uint64_t tbl_off;       // table arena offset (bytes)
    uint64_t out_off;       // compacted output offset (set by the scan)
    uint64_t out_size[2];   // encoded size per order (set after encode)
    uint64_t nwords[2];     // renorm words per order (set by the encoder)
    uint32_t states[2][kStates];
    int32_t mode;           // FQXV_RANS_ORDER0/1, BEST_TIE0/1
    int32_t nu;             // |U|: symbols present plus context 0 (order-1 tables)
    int32_t nctx;           // present order-1 contexts
    int32_t chosen;         // order written to the output
};

// One encode job: a (block, order) pair; the job list is sorted by size.
struct EncJob {
    uint32_t block;
    uint32_t order;
};

// Table arena layout per block (bytes from tbl_off):
//   [0, 2048)               order-0: 256 x uint2 {magic, (freq << 12) | cum}
//   [2048, 2048 + 256)      order-1: u8 dense index of each byte value (0xFF: not in U)
//   [2304, ...)             order-1: nu x nu x uint2, row = context, column = symbol
constexpr uint64_t kTblO0 = 0;
constexpr uint64_t kTblUmap = 2048;
constexpr uint64_t kTblO1 = 2304;
__host__ __device__ inline uint64_t enc_table_bytes(uint64_t n) {
    uint64_t u = n + 1 < 256 ? n + 1 : 256;
    return kTblO1 + u * u * 8;
}

// Polls of an mbarrier before a decode kernel gives up on a table copy and
// reports FQXV_RANS_E_TIMEOUT (several milliseconds; a copy lands in
// microseconds).
constexpr uint32_t kWaitPolls = 1u << 22;

// Decode-side descriptor of one stream.
struct DecStream {
    uint64_t src_off, src_len;   // input span
    uint64_t dst_off, dst_cap;   // output span
    uint64_t max_len;            // decode_bounded bound (UINT64_MAX: none)
    uint64_t n;                  // declared output length
    uint64_t words_off;          // absolute byte offset of the renorm words
    uint64_t words_len;          // bytes after the states
    uint64_t tbl_off;            // table arena offset (bytes)
    int32_t order;
    int32_t status;
    int32_t nctx;                // present order-1 contexts (K)
    int32_t ctx0;                // global format: dense index of context 0 (0xFF: absent)
    int32_t cls;                 // decode class (kClsO0, kClsO1Dense, kClsO1Global)
    int32_t nd;                  // dense format: |D| (symbols and contexts), DEAD = nd
    int32_t start;               // dense format: index of context 0 (DEAD when absent)
    uint32_t tbl_bytes;          // bytes of the table image staged into shared memory
    uint32_t tbl_bytes_planes;   // dense format with bit-plane columns: image + planes
                                 // (the four-warp decoder stages these); else tbl_bytes
    uint32_t states[kStates];
};

enum { kClsNone = 0, kClsO0 = 1, kClsO1Dense = 2, kClsO1Global = 3 };
// Launch classes of dense streams decoded by one warp each: |D| <=
// kSmallMaxNd (packed columns, chains stepped in registers) and wider
// alphabets (byte columns, up to five chains per lane). kClsO1Dense is the
// four-warp decoder of the byte columns.
constexpr int kClsO1Small = 4;
constexpr int kClsO1Wide = 5;
constexpr int kSmallMaxNd = 15;
// Up to this |D| every chain of a round has its own lane (3 |D| + 1 <= 31)
// and rows are resolved by shuffles; above it rows go through shared memory.
constexpr int kShflMaxNd = 10;

// Decode table arena per stream (bytes from tbl_off).
//   order-0: 4096 x u32 packed ((freq - 1) << 20) | ((slot - cum) << 8) | sym.
//   order-1 dense (|D| <= kDenseMax and an image of at most kDenseImageMax
//     bytes): D = present contexts and every symbol of their tables, in
//     ascending byte order; DEAD = |D| marks "absent context". The slot axis
//     is cut at every position where some context's symbol changes (a
//     boundary: a cum value of a present symbol); between two boundaries
//     every context decodes every slot to the same symbol, so one column per
//     boundary holds, for each context, the dense symbol of that slot range.
//     [0, 4096)                 M8: u8 per slot, the slot's column less the
//                               first column of its 256-slot block
//     [4096, 4160)              MB: u32 per 256-slot block, that first
//                               column (times S for byte columns: a byte
//                               offset)
//     [4160, + fc_bytes)        u32 (freq << 12) | cum, row = context, col = symbol
//     [.., + 256)               dense index -> byte value
//     [col_off, + ncol * S)     columns, S = dense_col_stride(nd) bytes each:
//                               byte d of column j = the dense symbol that
//                               context d decodes in column j's slots (DEAD
//                               for rows of absent contexts and for DEAD)
//     Full-range quality tables (|D| ~ 31) have ~480 columns: ~23 KB against
//     ~130 KB for a slot -> symbol table per context.
//     Packed form, |D| <= kSmallMaxNd: MB holds plain column indices, and the
//     columns are u64 at col_off, entry d in bits [4d, 4d + 4), so a chain
//     step is a shift of a register instead of a shared-memory load.
//   order-1 global (more symbols, or more columns than the image holds):
//     [256 B] raw context -> dense index (0xFF absent), then per present
//     context t: 4096 x u16 (sym << 8) | dense(sym), then 256 x u32
//     (freq << 12) | cum.
constexpr int kDenseMax = 47;
constexpr uint32_t kDenseMB = 4096;          // M8: u8 per slot
constexpr uint32_t kDenseM = kDenseMB + 64;  // MB: u32 per 256-slot block
constexpr uint32_t kDenseImageMax = 160 * 1024;
__host__ __device__ inline uint32_t dense_col_stride(int nd) { return (uint32_t)((nd + 1 + 15) / 16 * 16); }
__host__ __device__ inline uint32_t dense_fc_bytes(int nd) {
    return (uint32_t)(((nd + 1) * (nd + 1) * 4 + 15) / 16 * 16);
}
__host__ __device__ inline uint32_t dense_col_off(int nd) { return kDenseM + dense_fc_bytes(nd) + 256; }
__host__ __device__ inline bool dense_packed(int nd) { return nd <= kSmallMaxNd; }
// Bytes of the table image (what is staged into shared memory).
__host__ __device__ inline uint32_t dense_table_bytes(int nd, uint32_t ncol) {
    return dense_packed(nd) ? dense_col_off(nd) + (8 * ncol + 15) / 16 * 16
                            : dense_col_off(nd) + ncol * dense_col_stride(nd);
}
// Bit-plane columns, kSmallMaxNd < |D| <= kPlaneMaxNd: after the byte
// columns, column j's entries as five u32 planes at j * 32 (plane p, bit c =
// bit p of the entry of context c, rotated left by p; three words of
// padding), so that a chain step is five funnel shifts and four bit selects
// in registers instead of a shared-memory load. The planes offset is
// dense_table_bytes, and column j's planes sit at the byte offset of its byte
// column (the byte stride is 32 for these |D|).
constexpr int kPlaneMaxNd = 31;
constexpr uint32_t kPlaneStride = 32;
__host__ __device__ inline bool dense_planes(int nd) { return nd > kSmallMaxNd && nd <= kPlaneMaxNd; }
// Bytes the parse needs in the arena while building the image: the packed
// form is built from byte columns placed after it.
__host__ __device__ inline uint32_t dense_build_bytes(int nd, uint32_t ncol) {
    return dense_packed(nd) ? dense_table_bytes(nd, ncol) + ncol * dense_col_stride(nd)
                            : dense_table_bytes(nd, ncol);
}
constexpr uint64_t kDecCtxMap = 0;
constexpr uint64_t kDecO1Base = 256;
constexpr uint64_t kDecO1Slot = 4096 * 2;
constexpr uint64_t kDecO1Fc = 256 * 4;
constexpr uint64_t kDecO1Ctx = kDecO1Slot + kDecO1Fc;
__host__ __device__ inline uint64_t dec_table_bytes(uint64_t src_len) {
    // A stream with K order-1 tables is at least 41 + 512 K bytes long.
    uint64_t k = src_len > 41 ? (src_len - 41) / 512 : 0;
    if (k > 256) k = 256;
    uint64_t b = 16384;
    if (k > 0) {
        const uint64_t g = kDecO1Base + k * kDecO1Ctx;
        b = g > b ? g : b;
        b = kDenseImageMax > b ? kDenseImageMax : b;
    }
    return b;
}

// Shared-memory layout of the decode kernels.
constexpr uint32_t kRingBytes = 2048;       // renorm-word ring, 4 x 512 B segments
constexpr uint32_t kOutRows = 3 * kDenseMax + 1;

inline uint64_t align_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

// ---- launchers (rans_encode.cu / rans_decode.cu) ---------------------------
// `grid` clusters of `cluster` CTAs (1..8) over the blocks order[0, nblocks);
// returns the launch status. `keys` (nullable, u16 per input byte) receives
// each position's order-1 table index for the encode.
cudaError_t launch_enc_model(const uint8_t *src, EncBlock *blocks, const uint32_t *order, int nblocks,
                             uint8_t *tbl, uint32_t *hist_scratch, uint16_t *keys, int grid, int cluster,
                             cudaStream_t s);
void launch_enc_run(const uint8_t *src, EncBlock *blocks, const EncJob *jobs, int njobs,
                    const uint8_t *tbl, uint16_t *words, int *queue, const uint16_t *keys, int grid,
                    cudaStream_t s);
void launch_enc_select_scan(EncBlock *blocks, int nblocks, uint64_t *total, cudaStream_t s);
void launch_enc_pack(EncBlock *blocks, int nblocks, const uint8_t *tbl, const uint16_t *words,
                     uint8_t *dst, int grid, cudaStream_t s);

void launch_dec_parse(const uint8_t *src, DecStream *streams, int nstreams, uint8_t *tbl,
                      int grid, cudaStream_t s);
// Runs the decode of the streams listed in `list` (all of class `cls`);
// smem_bytes is the dynamic shared memory of the class (largest member).
// `mirror` (nullable): each stream decoded without error is also copied to
// mirror + dst_off (the device alias of a pinned host destination) by the
// CTA that decoded it.
void launch_dec_run(int cls, const uint8_t *src, DecStream *streams, const uint32_t *list, int nlist,
                    const uint8_t *tbl, uint8_t *dst, int *queue, int grid, uint32_t smem_bytes,
                    uint32_t first_polls, uint8_t *mirror, cudaStream_t s);
// `nd`: the largest |D| among the launch's streams (the one-warp wide
// decoder keeps its rows, 3 |D| + 2 per buffer, in dynamic shared memory).
uint32_t dec_smem_bytes(int cls, uint32_t tbl_bytes, int nd = kDenseMax);
// Bytes of the one-warp wide decoder's two row buffers for |D| = nd.
__host__ __device__ inline uint32_t wide_rows_bytes(int nd) { return (uint32_t)((2 * (3 * nd + 2) * 16 + 127) / 128 * 128); }
// Dynamic shared memory with which one CTA of a decode class fills an SM (no
// other CTA fits beside it); 0 when the class cannot.
// per_sm > 1: the share that lets exactly per_sm such CTAs fill an SM.
uint32_t dec_exclusive_smem(int cls, int per_sm = 1);
// CTAs of a decode class that fit on one SM with `smem_bytes` of dynamic
// shared memory (registers and static shared memory included).
int dec_blocks_per_sm(int cls, uint32_t smem_bytes);

int sm_count(int device);

}  // namespace fqxv
