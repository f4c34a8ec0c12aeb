// Internal definitions of the CRC-32C / block-frame kernels
// (frame_kernels.cu) and their C-ABI (frame_capi.cu). Not part of the ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/fqxv_frame_gpu.h"

namespace fqxv {

// crates/fqxv/src/container/format.rs:71-99
constexpr uint64_t kFrameHead = 16;                  // "FQXB" + u64 len + u32 crc
constexpr uint64_t kFrameTerm = 12;                  // "FQXB" + u64 0
constexpr uint64_t kMaxBlockPayload = 1ull << 31;    // MAX_BLOCK_SEQ_BYTES (256 MiB) x 8

// Piece kernel shape: one CTA per SM (the tables take 128 KiB of shared
// memory); a warp keeps up to 2 x kCrcUnroll lines of loads in flight. The
// frame copy also holds the realigned words and moves twice the bytes: it
// runs 768 threads so each may keep 80 registers, 2 x kCopyUnroll lines.
constexpr int kCrcThreads = 1024;
constexpr int kCrcUnroll = 12;
constexpr int kCopyThreads = 768;
constexpr int kCopyUnroll = 12;
// Piece size 2^shift: about kCrcPieceTarget pieces per pass (four per warp
// slot of 148 SMs x 32 warps), between 32 KiB and 256 KiB.
constexpr int kCrcMinShift = 15;
constexpr int kCrcMaxShift = 18;
constexpr uint32_t kCrcPieceTarget = 16384;

// Frame walk: frames walked by one thread before the marker scan takes over,
// and the most marker hits the chain kernel ranks in shared memory.
constexpr uint32_t kWalkHops = 32;
constexpr uint32_t kChainMax = 8192;
// key u64, plen u32, crc u32, succ / jump / rank u16, kind u8 per hit
constexpr uint32_t kChainSmem = kChainMax * (8 + 4 + 4 + 2 + 2 + 2 + 1);

// Job header in device memory (first bytes of the target arena).
struct FrameJob {
    uint32_t ntargets;
    uint32_t npieces;
    uint32_t counter;       // unused by the piece kernel (static schedule); reset
    int32_t piece_shift;
    uint32_t nframes;       // frame walk: entries written
    int32_t terminated;     // frame walk: terminator frame seen
    uint64_t consumed;      // frame walk: bytes walked
    uint64_t walk_pos;      // frame walk: where the serial walk stopped
    uint32_t walk_done;     // frame walk: 1 once the walk is over
    uint32_t ncand;         // frame walk: marker hits found by the scan
    uint32_t cand_overflow; // frame walk: more hits than kChainMax
    uint32_t pad;
};

// A marker hit of the frame scan: position and the 12 bytes after the marker.
struct WalkCand {
    uint64_t pos;
    uint64_t plen;
    uint32_t crc;
    uint32_t pad;
};

// One CRC target: bytes [src_off, src_off + len) of the source (and, for a
// frame copy, their place dst_off in the destination).
struct CrcTarget {
    uint64_t src_off;
    uint64_t len;
    uint64_t dst_off;
    uint64_t piece_base;    // index of the target's first piece
};

// One piece: bytes [src, src + len) of the source (copied to dst for a
// frame copy) of target `target`; mult = x^(8 k) mod P, k the target's bytes
// after the piece.
struct CrcPiece {
    uint64_t src;
    uint64_t dst;
    uint32_t len;
    uint32_t target;
    uint32_t mult;
    uint32_t pad;
};

// One frame of a walk (block.rs:1209-1254).
struct WalkEntry {
    uint64_t pay_off;
    uint64_t pay_len;
    uint32_t stored_crc;
    uint32_t crc;
    int32_t status;
    uint32_t target;        // CRC target index, ~0 for a structural failure
};

struct PayloadRef {
    uint64_t off;
    uint64_t len;
};

__host__ __device__ inline int crc_piece_shift(uint64_t total, uint32_t target, int min_shift, int max_shift) {
    const uint64_t want = total / target;
    int s = min_shift;
    while (s < max_shift && (1ull << s) < want) s++;
    return s;
}

// Pieces of a target of `len` bytes starting at address `addr` (pieces are
// cut at multiples of 2^shift of the address).
__host__ __device__ inline uint64_t crc_piece_count(uint64_t addr, uint64_t len, int shift) {
    if (len == 0) return 0;
    const uint64_t a0 = addr & ((1ull << shift) - 1);
    return ((a0 + len - 1) >> shift) + 1;
}

cudaError_t launch_crc_plan(FrameJob *job, CrcTarget *targets, CrcPiece *pieces, uint32_t *crc_out,
                            uint32_t ntargets_hint, uint64_t align_base, int by_dst, int sms, cudaStream_t s);
cudaError_t launch_crc_pieces(const uint8_t *src, uint8_t *dst, FrameJob *job, const CrcPiece *pieces,
                              uint32_t *crc_out, int copy, int grid, cudaStream_t s);
cudaError_t launch_frame_heads(uint8_t *dst, const FrameJob *job, const CrcTarget *targets,
                               const uint32_t *crc_out, uint32_t n, uint64_t term_off, cudaStream_t s);
// The walk, the marker scan, the chain and the piece bases (four launches).
cudaError_t launch_frame_walk(const uint8_t *src, uint64_t len, uint32_t max_frames, FrameJob *job,
                              CrcTarget *targets, WalkEntry *walk, WalkCand *cand, uint64_t align_base, int sms,
                              cudaStream_t s);
cudaError_t launch_frame_verify(const FrameJob *job, WalkEntry *walk, const uint32_t *crc_out, uint32_t max_frames,
                                cudaStream_t s);
cudaError_t launch_stream_locs(const uint8_t *src, const PayloadRef *payloads, uint32_t n, FrameJob *job,
                               CrcTarget *targets, int32_t *status, uint64_t align_base, cudaStream_t s);

}  // namespace fqxv
