/*
 * fqxv_streams_gpu.h -- the coder's other in-container callers, batched on the
 * B200 coder:
 *
 *   put_stream / get_stream   crates/fqxv-lroverlap/src/codec.rs:289-363
 *       -> fqxv_put_streams_host / fqxv_get_streams_host
 *   the reorder permutation's byte planes
 *       crates/fqxv/src/container/reorder.rs:597-609 (encode_perm),
 *       :1089-1105 (decode_permutation)
 *       -> fqxv_perm_encode_host / fqxv_perm_decode_host
 *
 * A put_stream frame is [varint raw_len] then, when raw_len > 0,
 * [varint enc_len][rANS stream], the stream the smaller of the two orders with
 * ties to order-1. The permutation is n u32 split into four byte planes
 * (plane k = byte k of every entry) coded as one stream, the smaller order
 * with ties to order-0. Host buffers; synchronous; contexts as in
 * fqxv_rans_gpu.h.
 */
#ifndef FQXV_STREAMS_GPU_H
#define FQXV_STREAMS_GPU_H

#include "fqxv_rans_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

enum {
    /* fqxv_lroverlap::Error::Corrupt "malformed lroverlap block" (lib.rs:116-118) */
    FQXV_STREAM_E_CORRUPT = 64,
    /* fqxv::Error::Malformed("bad permutation") (reorder.rs:1097-1098) */
    FQXV_PERM_E_BAD = 65,
    /* fqxv::Error::Malformed("permutation length mismatch") (reorder.rs:1099-1101) */
    FQXV_PERM_E_LENGTH = 66
};

/* put_stream for n raw streams (spans of h_src), in one coding pass: frame i
 * goes to h_dst at out[i], frames back to back in order. *needed (may be NULL)
 * receives the bytes all frames take; if that exceeds cap nothing is written
 * and FQXV_RANS_E_DST_TOO_SMALL is returned. */
int fqxv_put_streams_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, const fqxv_rans_span *raw, size_t n,
                          uint8_t *h_dst, uint64_t cap, fqxv_rans_span *out, uint64_t *needed);

/* get_stream n times from h_src[pos, len), in one decoding pass: stream i's
 * bytes go to h_dst at out[i] (back to back), status[i] is OK or
 * FQXV_STREAM_E_CORRUPT (bad framing, an undecodable stream, or a length other
 * than the frame's raw_len). The frames after the first failing one are not
 * read (status CORRUPT, empty). *end_pos receives the position after the last
 * frame read. *needed (may be NULL) receives the output bytes; if that
 * exceeds cap nothing is written and FQXV_RANS_E_DST_TOO_SMALL is returned.
 * Returns the first non-OK status, or OK. */
int fqxv_get_streams_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, uint64_t len, uint64_t pos, size_t n,
                          uint8_t *h_dst, uint64_t cap, fqxv_rans_span *out, int32_t *status, uint64_t *end_pos,
                          uint64_t *needed);

/* encode_perm: the n entries of order split into four byte planes on the GPU
 * and coded there; the stream (at most 649 + 8 n bytes) goes to h_dst,
 * *out_len its length. */
int fqxv_perm_encode_host(fqxv_rans_ctx *ctx, const uint32_t *order, uint64_t n, uint8_t *h_dst, uint64_t cap,
                          uint64_t *out_len);

/* decode_permutation: the stream h_src[0, len) decoded (bounded by 4 n) and
 * its byte planes joined on the GPU into order[0, n). FQXV_PERM_E_BAD for any
 * decode failure, FQXV_PERM_E_LENGTH when it does not hold exactly 4 n
 * bytes. */
int fqxv_perm_decode_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, uint64_t len, uint64_t n, uint32_t *order);

#ifdef __cplusplus
}
#endif
#endif
