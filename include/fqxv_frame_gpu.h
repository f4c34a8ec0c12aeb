/*
 * fqxv_frame_gpu.h -- C ABI of the B200 CRC-32C and container block frames.
 *
 * The byte arithmetic of crates/fqxv/src/crc.rs and the block framing of
 * crates/fqxv/src/container/block.rs, batched on the GPU:
 *
 *   crc32c(bytes)                 crc.rs:74      -> fqxv_crc32c_batch
 *   crc32c_combine(a, b, len_b)   crc.rs:116     -> fqxv_crc32c_combine
 *   write_blocks frames           block.rs:110   -> fqxv_frame_blocks
 *   read_block, frame by frame    block.rs:1209  -> fqxv_read_blocks
 *   payload_stream_locs           block.rs:961   -> fqxv_payload_stream_locs
 *
 * CRC-32C: reflected polynomial 0x82F63B78, init and xor-out 0xFFFFFFFF
 * (check value 0xE3069283 over "123456789"). A frame is
 * [4 "FQXB"][u64 payload_len LE][u32 crc32c(payload) LE][payload]; a frame of
 * length 0 ends the block region.
 *
 * Contexts, spans and status codes are those of fqxv_rans_gpu.h; calls on one
 * context are serialised, and every call is synchronous.
 */
#ifndef FQXV_FRAME_GPU_H
#define FQXV_FRAME_GPU_H

#include "fqxv_rans_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Frame status codes (crates/fqxv/src/lib.rs:167-178 Error variants); their
 * text comes from fqxv_rans_status_message. */
enum {
    /* Error::Truncated "truncated fqxv stream": a frame's length, CRC or
     * payload runs past the end of the buffer, or a payload is too short for
     * its stream lengths. */
    FQXV_FRAME_E_TRUNCATED = 32,
    /* Error::Corrupt { what: "block {i}" }: the payload's CRC-32C differs. */
    FQXV_FRAME_E_CORRUPT = 33,
    /* Error::Corrupt { what: "block {i} (bad sync marker)" }. */
    FQXV_FRAME_E_BAD_SYNC = 34,
    /* Error::Malformed("block payload length exceeds the maximum"):
     * declared length above MAX_BLOCK_PAYLOAD (2 GiB, format.rs:87). */
    FQXV_FRAME_E_TOO_LARGE = 35
};

#define FQXV_FRAME_HEAD_LEN 16u /* format.rs:99 FRAME_HEAD_LEN */
#define FQXV_FRAME_TERM_LEN 12u /* "FQXB" + u64 0 */

/* CRC-32C of each span of device buffer d_src (spans on the host) into the
 * host array crcs. Empty spans give 0. crc.rs:74. */
int fqxv_crc32c_batch(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *spans, size_t n,
                      uint32_t *crcs);
/* The same over a host buffer (copied to the device first). */
int fqxv_crc32c_batch_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, const fqxv_rans_span *spans, size_t n,
                           uint32_t *crcs);

/* crc.rs:116: crc32c(A ++ B) from crc32c(A), crc32c(B) and |B|. Arithmetic
 * on the three values only (no buffer, no device). */
uint32_t fqxv_crc32c_combine(uint32_t crc_a, uint32_t crc_b, uint64_t len_b);

/* Bytes fqxv_frame_blocks writes: 16 + length per payload, + 12 with the
 * terminator. */
uint64_t fqxv_frame_blocks_bound(const fqxv_rans_span *payloads, size_t n, int terminate);

/* block.rs:110-142: frame the n payloads of device buffer d_src (spans on the
 * host) back to back into d_dst (device, capacity dst_cap; must not overlap
 * d_src); terminate != 0 appends the zero-length terminator frame. Each
 * payload is copied and checksummed in one pass. frame_offsets[i] (host, may
 * be NULL) receives frame i's offset in d_dst, crcs[i] (host, may be NULL) the
 * payload's CRC-32C, *total (may be NULL) the bytes written. A zero-length
 * payload is framed as given (a reader takes it for the terminator, as the
 * reference's does). */
int fqxv_frame_blocks(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *payloads, size_t n,
                      int terminate, uint8_t *d_dst, uint64_t dst_cap, uint64_t *frame_offsets, uint32_t *crcs,
                      uint64_t *total);
/* The same with host buffers for the payloads and the frames. */
int fqxv_frame_blocks_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, const fqxv_rans_span *payloads, size_t n,
                           int terminate, uint8_t *h_dst, uint64_t dst_cap, uint64_t *frame_offsets,
                           uint32_t *crcs, uint64_t *total);

/* block.rs:1209-1254 applied frame after frame from offset 0 of d_src[0, len)
 * (device). Stops at a clean end (fewer than 4 bytes left), at the
 * terminator (*terminated = 1, its 12 bytes consumed), after max_frames
 * frames, or at a structural failure: bad marker (BAD_SYNC), short length,
 * CRC or payload (TRUNCATED), or a declared length above 2 GiB (TOO_LARGE);
 * that frame's entry carries the status and payloads[i] = {frame offset, 0}.
 * Every frame that passed the structural checks has its payload CRC-32C
 * verified on the GPU (CORRUPT on a mismatch; the walk goes on past it).
 * Host outputs: payloads[i] (payload span), crcs[i] (computed CRC), status[i]
 * for i < *nframes; *consumed = bytes walked. Returns the first non-OK status
 * in frame order (the error the reference's reader stops at), or OK. */
int fqxv_read_blocks(fqxv_rans_ctx *ctx, const uint8_t *d_src, uint64_t len, size_t max_frames,
                     fqxv_rans_span *payloads, uint32_t *crcs, int32_t *status, size_t *nframes, uint64_t *consumed,
                     int *terminated);
/* The same over a host buffer (copied to the device first). */
int fqxv_read_blocks_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, uint64_t len, size_t max_frames,
                          fqxv_rans_span *payloads, uint32_t *crcs, int32_t *status, size_t *nframes,
                          uint64_t *consumed, int *terminated);

/* format.rs:252-266 StreamLoc. */
typedef struct fqxv_stream_loc {
    uint64_t offset;
    uint32_t len;
    uint32_t crc;
} fqxv_stream_loc;

/* block.rs:961-980 for n plain payloads of device buffer d_src (spans on the
 * host): each payload is [24 digests][u32 n_reads]([u32 len][bytes]) x 3, and
 * locs[3i + s] (host) receives stream s's (offset, len, crc32c), the offset
 * being base + the stream's offset in d_src (pass the archive position of
 * d_src[0] as base to get the reference's absolute offsets). status[i]
 * (host) is OK or FQXV_FRAME_E_TRUNCATED (locs then zero). Returns the first
 * non-OK status, or OK. */
int fqxv_payload_stream_locs(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *payloads, size_t n,
                             uint64_t base, fqxv_stream_loc *locs, int32_t *status);

#ifdef __cplusplus
}
#endif
#endif
