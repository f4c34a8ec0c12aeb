/*
 * CPU oracle for the fqxv-rans Nx16 coder -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference crate `crates/fqxv-rans`:
 *   model.rs  -- constants, normalize, from_freqs validation, EncSym
 *   scalar.rs -- byte format, order-0 / order-1 encode and decode, errors
 *   lib.rs    -- decode_bounded / peek_output_len
 *   avx2.rs, avx512.rs -- the order-0 SIMD encode/decode (rans_simd.c)
 *
 * Only the test suite, the smoke check and the benchmark's CPU-baseline leg
 * may load this library, and only as the checker / the timed CPU path. The
 * product (libfqxv_rans_gpu.so) never links or calls it.
 *
 * Parity pin: decoding the 32 order-0 rANS streams stored in the reference's
 * container fixtures and re-encoding them reproduces the stored bytes exactly
 * (tests/golden). Order-1 has no stored bytes in the reference; its pin is
 * this restatement of scalar.rs:61-111 / :180-217.
 *
 * Status codes share their numeric values with include/fqxv_rans_gpu.h.
 */
#ifndef FQXV_RANS_ORACLE_H
#define FQXV_RANS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ORC_OK = 0,
    ORC_E_TRUNCATED = 1,         /* "truncated stream"                  scalar.rs:261 */
    ORC_E_UNKNOWN_ORDER = 2,     /* "unknown order tag"                 scalar.rs:153 */
    ORC_E_FREQ_EXCEEDS = 3,      /* "rANS freq table exceeds TOTFREQ"   model.rs:165 */
    ORC_E_FREQ_SUM = 4,          /* "... does not sum to TOTFREQ"       model.rs:169 */
    ORC_E_ABSENT_CONTEXT = 5,    /* "symbol references absent context"  scalar.rs:206 */
    ORC_E_ALLOC = 6,             /* "rANS output length too large to allocate" model.rs:202 */
    ORC_E_BOUND = 7,             /* "rANS output length exceeds caller bound" lib.rs:228 */
    ORC_E_TRUNCATED_RENORM = 8,  /* "truncated renorm stream"           avx2.rs:207 */
    ORC_E_X_MALFORMED = 9,       /* extended format only (rans_x.c): inconsistent transform data */
    ORC_E_INVALID_ARG = 16,
    ORC_E_DST_TOO_SMALL = 17,
    /* container frames (crates/fqxv/src/lib.rs:167-178, block.rs:1209-1254) */
    ORC_FRAME_E_TRUNCATED = 32,  /* Error::Truncated "truncated fqxv stream" */
    ORC_FRAME_E_CORRUPT = 33,    /* Error::Corrupt "block {i}" (crc mismatch) */
    ORC_FRAME_E_BAD_SYNC = 34,   /* Error::Corrupt "block {i} (bad sync marker)" */
    ORC_FRAME_E_TOO_LARGE = 35   /* Error::Malformed("block payload length exceeds the maximum") */
};

/* model.rs:9-19 */
#define ORC_SCALE_BITS 12u
#define ORC_TOTFREQ 4096u
#define ORC_RANS_L 65536u
#define ORC_N_STATES 32

/* Worst-case encoded size: header + tables + states + one u16 per symbol. */
size_t orc_encode_bound(size_t n, int order);

/* model.rs:213-264 */
void orc_normalize(const uint32_t counts[256], uint16_t freq[256]);

/* model.rs:160-174: 0, ORC_E_FREQ_EXCEEDS or ORC_E_FREQ_SUM. */
int orc_validate_freqs(const uint16_t freq[256]);

/* model.rs:70-133: the encode map `(v / f) << 12 + v % f + c` through the
 * reference's reciprocal-or-division split. Exposed for the exhaustive test. */
uint32_t orc_encsym_apply(uint32_t freq, uint32_t cum, uint32_t v);
/* avx2.rs:245-264 / :385-393: the same map by magic multiply + one correction. */
uint32_t orc_magic_apply(uint32_t freq, uint32_t cum, uint32_t v);

/* scalar.rs:29-55 (order 0) and :61-111 (order 1). Returns status; the
 * stream length in *out_len. `dst_cap` must be >= orc_encode_bound(n, order). */
int orc_encode(const uint8_t *src, size_t n, int order, uint8_t *dst, size_t dst_cap,
               size_t *out_len);

/* lib.rs:207: 0 and *n, or ORC_E_TRUNCATED when shorter than 9 bytes. */
int orc_peek_output_len(const uint8_t *src, size_t len, uint64_t *n);

/* scalar.rs:143-238. The output length `n` from the header is written to
 * *out_len on success. A stream declaring n > dst_cap fails with ORC_E_ALLOC
 * at the point the reference allocates (after the tables and states parse). */
int orc_decode(const uint8_t *src, size_t len, uint8_t *dst, size_t dst_cap, size_t *out_len);

/* lib.rs:226-231. */
int orc_decode_bounded(const uint8_t *src, size_t len, size_t max_len, uint8_t *dst,
                       size_t dst_cap, size_t *out_len);

/* model.rs:313-365 sweep; returns the mismatch count (0 = exact). */
size_t orc_check_apply_sweep(void);

/* ---- SIMD restatements (rans_simd.c): order-0 only, byte-identical ---- */
/* 0 = scalar only, 1 = AVX2, 2 = AVX-512F (runtime CPU detection). */
int orc_simd_level(void);
/* avx2.rs:269-307 / avx512.rs:164-198; level 1 = AVX2, 2 = AVX-512. */
int orc_encode_o0_simd(int level, const uint8_t *src, size_t n, uint8_t *dst, size_t dst_cap,
                       size_t *out_len);
/* avx2.rs:58-105 / avx512.rs:29-75. */
int orc_decode_o0_simd(int level, const uint8_t *src, size_t len, uint8_t *dst,
                       size_t dst_cap, size_t *out_len);

/* ---- The reference's dispatch (lib.rs:111-127, :186-200) ----
 * encode: order-0 -> widest SIMD encoder, order-1 -> scalar.
 * decode: order-0 tag -> widest SIMD decoder, else scalar. */
int orc_encode_dispatch(const uint8_t *src, size_t n, int order, uint8_t *dst, size_t dst_cap,
                        size_t *out_len);
int orc_decode_dispatch(const uint8_t *src, size_t len, uint8_t *dst, size_t dst_cap,
                        size_t *out_len);

/* ---- Block-parallel batch (the reference's rayon-over-blocks shape,
 * crates/fqxv/src/container/decompress.rs:46-52), for the CPU baseline.
 * Blocks are [src + src_off[i], src_len[i]); outputs at dst + dst_off[i]
 * with capacity dst_cap[i]; per-block length and status returned.
 * order: 0, 1, or 2 = both orders, keep the smaller (ties -> order 0,
 * crates/fqxv-tokenizer/src/lib.rs:91-95). nthreads <= 0 = all cores. */
int orc_encode_batch(const uint8_t *src, const uint64_t *src_off, const uint64_t *src_len,
                     size_t nblocks, int order, uint8_t *dst, const uint64_t *dst_off,
                     const uint64_t *dst_cap, uint64_t *out_len, int32_t *status, int nthreads);
int orc_decode_batch(const uint8_t *src, const uint64_t *src_off, const uint64_t *src_len,
                     size_t nblocks, uint8_t *dst, const uint64_t *dst_off,
                     const uint64_t *dst_cap, uint64_t *out_len, int32_t *status, int nthreads);

/* ---- Extended stream format (rans_x.c): PARITY UNPINNED -------------------
 * A new format tag (first byte 0x80 | flags) with no counterpart in the
 * reference: 4-way interleaved cores and the STRIPE / RLE / PACK / CAT
 * transforms. Layout in rans_x.c. */
enum {
    ORC_X_ORDER1 = 0x01,
    ORC_X_N4 = 0x02,
    ORC_X_STRIPE = 0x04,
    ORC_X_RLE = 0x08,
    ORC_X_PACK = 0x10,
    ORC_X_CAT = 0x20,
    ORC_X_ALL = 0x3f
};
/* Cores: nstates 32 is the reference stream (orc_encode); 4 writes tag
 * 2 | order with four states. Decode takes either. */
size_t orc_core_bound(size_t n, int order, int nstates);
int orc_core_encode(const uint8_t *src, size_t n, int order, int nstates, uint8_t *dst, size_t *out_len);
int orc_core_decode(const uint8_t *src, size_t len, uint8_t *dst, size_t cap, size_t *out_len);
size_t orc_x_encode_bound(size_t n, int flags);
int orc_x_encode(const uint8_t *src, size_t n, int flags, uint8_t *dst, size_t dst_cap, size_t *out_len);
/* Decodes an extended stream, or a reference stream (first byte < 0x80). */
int orc_x_decode(const uint8_t *src, size_t len, uint8_t *dst, size_t dst_cap, size_t *out_len);
/* The selection over reference and extended candidates (rans_x.c); *cand
 * receives the winning candidate's index. */
size_t orc_x_best_bound(size_t n);
int orc_x_encode_best(const uint8_t *src, size_t n, uint8_t *dst, size_t dst_cap, size_t *out_len, int *cand);
/* Blocks in parallel on all host cores: encode with `flags` (0x40: the
 * selection; choice[i] gets the candidate) or, with decode != 0, decode. */
int orc_x_batch(const uint8_t *src, const uint64_t *src_off, const uint64_t *src_len, size_t nblocks, int flags,
                int decode, uint8_t *dst, const uint64_t *dst_off, const uint64_t *dst_cap, uint64_t *out_len,
                int32_t *status, int32_t *choice, int nthreads);

/* ---- CRC-32C and block frames (frame_oracle.c) ------------------------
 * crates/fqxv/src/crc.rs and crates/fqxv/src/container/block.rs. */
#define ORC_FRAME_HEAD 16u                     /* format.rs:99 FRAME_HEAD_LEN */
#define ORC_FRAME_TERM 12u                     /* "FQXB" + u64 0 */
#define ORC_MAX_BLOCK_PAYLOAD (1ull << 31)     /* format.rs:87 (256 MiB x 8) */
uint32_t orc_crc32c(const uint8_t *p, size_t n);
uint32_t orc_crc32c_update(uint32_t state, const uint8_t *p, size_t n);
uint32_t orc_crc32c_combine(uint32_t crc_a, uint32_t crc_b, uint64_t len_b);
int orc_frame_blocks(const uint8_t *src, const uint64_t *off, const uint64_t *len, size_t n, int terminate,
                     uint8_t *dst, uint64_t cap, uint64_t *frame_off, uint32_t *crcs, uint64_t *total);
int orc_read_blocks(const uint8_t *src, uint64_t len, size_t max_frames, uint64_t *pay_off, uint64_t *pay_len,
                    uint32_t *crcs, int32_t *status, size_t *nframes, uint64_t *consumed, int *terminated);
int orc_crc32c_batch(const uint8_t *src, const uint64_t *off, const uint64_t *len, size_t n, uint32_t *out,
                     int nthreads);
int orc_payload_stream_locs(const uint8_t *payload, uint64_t len, uint64_t block_offset, uint64_t loc_off[3],
                            uint32_t loc_len[3], uint32_t loc_crc[3]);

#ifdef __cplusplus
}
#endif
#endif
