/*
 * fqxv_rans_x_gpu.h -- the extended stream format of libfqxv_rans_gpu.so.
 *
 * No counterpart in the reference: fqxv-rans writes one format only, 32
 * interleaved states behind a flag-less [u8 order][u64 n] header
 * (crates/fqxv-rans/src/model.rs:19, scalar.rs:8-20), and has no raw path
 * (docs/design/testing.md:141-143). This is a new format tag -- first byte
 * 0x80 | flags -- adding 4-way interleaved cores and the STRIPE / RLE / PACK /
 * CAT transforms; streams of the reference format are left unchanged and
 * still decode here. Its definition is oracle/rans_x.c (the layout is
 * described there and in the library's rans_x.cu); parity against the
 * reference is unpinned, since the reference has no such streams.
 *
 *   flags  FQXV_X_ORDER1  cores use the order-1 model (else order-0)
 *          FQXV_X_N4      cores use 4 interleaved states (else 32)
 *          FQXV_X_STRIPE  four nested streams of the byte planes i % 4
 *          FQXV_X_RLE     runs of run symbols become a literal and a length
 *          FQXV_X_PACK    alphabets of <= 16 symbols packed 2, 4 or 8 per byte
 *          FQXV_X_CAT     cores stored raw
 */
#ifndef FQXV_RANS_X_GPU_H
#define FQXV_RANS_X_GPU_H

#include <stddef.h>
#include <stdint.h>

#include "fqxv_rans_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

enum {
    FQXV_X_ORDER1 = 0x01,
    FQXV_X_N4 = 0x02,
    FQXV_X_STRIPE = 0x04,
    FQXV_X_RLE = 0x08,
    FQXV_X_PACK = 0x10,
    FQXV_X_CAT = 0x20,
    FQXV_X_ALL = 0x3f,
    /* encode mode: the smallest of the reference streams (order 0, 1) and the
     * extended candidates PACK, RLE, PACK+RLE (order 0 and 1 each), STRIPE
     * and CAT, ties to the earlier of them in that order */
    FQXV_X_BEST = 0x40
};

/* Largest stream any flags (FQXV_X_BEST included) can write for n bytes. */
uint64_t fqxv_rans_x_stream_bound(uint64_t n);
/* Sum of fqxv_rans_x_stream_bound over the blocks. */
uint64_t fqxv_rans_x_encode_bound(const fqxv_rans_span *blocks, size_t nblocks);

/* Encode `nblocks` blocks of the device arena d_src with `flags` (a
 * combination of the FQXV_X_* transform flags, or FQXV_X_BEST). Streams go
 * back to back in block order into d_dst; out_spans (host) receives their
 * places, out_choice (host, may be NULL) the candidate index FQXV_X_BEST
 * chose (0, 1: reference order-0 / order-1 stream; 2-7: PACK, PACK order-1,
 * RLE, RLE order-1, PACK+RLE, PACK+RLE order-1; 8: STRIPE; 9: CAT) or the
 * flags. FQXV_RANS_E_INVALID_ARG when PACK meets more than 16 symbols.
 * Synchronous. */
int fqxv_rans_x_encode_batch(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *blocks, size_t nblocks,
                             int flags, uint8_t *d_dst, uint64_t dst_cap, fqxv_rans_span *out_spans,
                             int32_t *out_choice);

/* Decode `nblocks` streams of d_src, extended or reference format, into
 * d_dst at out_spans (offset, capacity). Per-stream status and length in
 * status / out_lens (host); returns the first failing status. Statuses:
 * the reference's Malformed kinds, and FQXV_RANS_E_X_MALFORMED for transform
 * data that does not fit together. Synchronous. */
int fqxv_rans_x_decode_batch(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *blocks, size_t nblocks,
                             uint8_t *d_dst, const fqxv_rans_span *out_spans, uint64_t *out_lens, int32_t *status);

#ifdef __cplusplus
}
#endif
#endif
