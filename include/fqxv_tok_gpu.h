/*
 * fqxv_tok_gpu.h -- C ABI of the read-name tokenizer over the B200 rANS coder.
 *
 * A batched drop-in for crates/fqxv-tokenizer/src/lib.rs:
 *   encode(names) -> payload   lib.rs:482  -> fqxv_tok_encode_host
 *   decode(payload) -> names   lib.rs:543  -> fqxv_tok_decode_host
 * for many blocks of names per call. Names are split into role streams
 * (token counts, per-column ops, string lengths and bytes, numeric literals,
 * zero paddings, per-column numeric deltas), the op columns run-length coded
 * and the deltas cut into byte planes, exactly as the reference does; every
 * role stream of every block is then rANS-coded (both orders, the smaller
 * kept, ties to order-0: lib.rs:91-95) or decoded in one GPU pass. Each
 * block's payload is byte-identical to the reference's encode of the same
 * names, and decode returns the reference's names or its first error.
 *
 * Names and payloads are host buffers. Calls are synchronous and serialise
 * on the context like the other batch calls.
 */
#ifndef FQXV_TOK_GPU_H
#define FQXV_TOK_GPU_H

#include "fqxv_rans_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Error::Malformed(msg) of the tokenizer (lib.rs:40-50); the text is
 * "malformed name stream: <msg>" (fqxv_rans_status_message). rANS errors of
 * a role stream come through as the coder's statuses 1..8. */
enum {
    FQXV_TOK_E_VERSION = 48,        /* "unsupported version" */
    FQXV_TOK_E_TRUNCATED = 49,      /* "truncated" */
    FQXV_TOK_E_VARINT = 50,         /* "varint too long" */
    FQXV_TOK_E_RECORDS = 51,        /* "record count exceeds token stream" */
    FQXV_TOK_E_SYM_UNDERRUN = 52,   /* "op sym underrun" */
    FQXV_TOK_E_RUN_TOO_LONG = 53,   /* "op run too long" */
    FQXV_TOK_E_OPS_BOUND = 54,      /* "op columns exceed the stream bound" */
    FQXV_TOK_E_PLANE_LEN = 55,      /* "delta plane length mismatch" */
    FQXV_TOK_E_MATCH = 56,          /* "MATCH without prior token" */
    FQXV_TOK_E_STR_UNDERRUN = 57,   /* "string data underrun" */
    FQXV_TOK_E_PAD_UNDERRUN = 58,   /* "pad underrun" */
    FQXV_TOK_E_DELTA_UNDERRUN = 59, /* "delta underrun" */
    FQXV_TOK_E_DELTA_PRIOR = 60,    /* "DELTA without numeric prior" */
    FQXV_TOK_E_UNKNOWN_OP = 61      /* "unknown op" */
};

/* Encode nblocks blocks of names. h_names holds the name bytes; name_spans[i]
 * is name i (offset, length in h_names); blocks[b] = {first name index, name
 * count}. Payload b goes to h_dst at out[b] (back to back in block order).
 * *needed (may be NULL) receives the bytes all payloads take; if that exceeds
 * cap nothing is written and FQXV_RANS_E_DST_TOO_SMALL is returned. */
int fqxv_tok_encode_host(fqxv_rans_ctx *ctx, const uint8_t *h_names, const fqxv_rans_span *name_spans,
                         size_t nnames, const fqxv_rans_span *blocks, size_t nblocks, uint8_t *h_dst,
                         uint64_t cap, fqxv_rans_span *out, uint64_t *needed);

/* Decode nblocks payloads (spans of h_src). The names of all blocks go back
 * to back into h_names (capacity names_cap); name_spans (capacity spans_cap
 * entries) receives each name's place, blocks[b] = {first name index, count}
 * and status[b] the block's status (OK, a FQXV_TOK_E_* or a coder status; a
 * failed block has no names). *names_needed / *spans_needed (may be NULL)
 * receive the sizes all blocks need; if either exceeds its capacity nothing
 * is written and FQXV_RANS_E_DST_TOO_SMALL is returned. Returns the first
 * non-OK block status, or OK. */
int fqxv_tok_decode_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, const fqxv_rans_span *payloads, size_t nblocks,
                         uint8_t *h_names, uint64_t names_cap, fqxv_rans_span *name_spans, uint64_t spans_cap,
                         fqxv_rans_span *blocks, int32_t *status, uint64_t *names_needed, uint64_t *spans_needed);

#ifdef __cplusplus
}
#endif
#endif
