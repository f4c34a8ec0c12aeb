/*
 * CPU restatement of the reference's CRC-32C and block-frame code -- TEST
 * INFRASTRUCTURE ONLY (the checker of the GPU frame path; never shipped).
 *
 *   crates/fqxv/src/crc.rs:19-37     byte-wise table of the reflected
 *                                    Castagnoli polynomial 0x82F63B78
 *   crc.rs:42-79                     Hasher / crc32c: init and xor-out ~0
 *   crc.rs:87-161                    crc32c_combine over GF(2) operators
 *   crates/fqxv/src/container/block.rs:110-142    write_blocks framing
 *   block.rs:961-980                 payload_stream_locs
 *   block.rs:1209-1254               read_block, walked over a buffer
 *
 * Parity is pinned by the CRC-32C check values of crc.rs:201-205 and by the
 * CRCs stored in the reference's golden archives
 * (the .fqxv files of crates/fqxv/tests/fixtures: header, block frames, reorder frames,
 * footer stream locations, whole-file and footer CRCs).
 */
#include "rans_oracle.h"

#include <string.h>

#define ORC_CRC_POLY 0x82F63B78u

static uint32_t crc_table[256];
static int crc_table_ready;

/* crc.rs:19-37: entry i is i run through eight shift-and-reduce steps. */
static void crc_table_init(void) {
    if (crc_table_ready) return;
    for (uint32_t i = 0; i < 256; i++) {
        uint32_t c = i;
        for (int k = 0; k < 8; k++) c = (c & 1) ? (c >> 1) ^ ORC_CRC_POLY : c >> 1;
        crc_table[i] = c;
    }
    crc_table_ready = 1;
}

/* crc.rs:55-61: Hasher::update over the running (un-finalised) state. */
uint32_t orc_crc32c_update(uint32_t state, const uint8_t *p, size_t n) {
    crc_table_init();
    for (size_t i = 0; i < n; i++) state = crc_table[(state ^ p[i]) & 0xFF] ^ (state >> 8);
    return state;
}

/* crc.rs:74-78 */
uint32_t orc_crc32c(const uint8_t *p, size_t n) { return orc_crc32c_update(0xFFFFFFFFu, p, n) ^ 0xFFFFFFFFu; }

/* crc.rs:87-99: column-operator times vector. */
static uint32_t op_apply(const uint32_t op[32], uint32_t v) {
    uint32_t r = 0;
    for (int i = 0; v; i++, v >>= 1)
        if (v & 1) r ^= op[i];
    return r;
}

/* crc.rs:102-106: square an operator. */
static void op_square(uint32_t dst[32], const uint32_t src[32]) {
    for (int i = 0; i < 32; i++) dst[i] = op_apply(src, src[i]);
}

/* crc.rs:116-161: crc32c(A ++ B) from crc32c(A), crc32c(B) and |B|. The
 * one-zero-bit operator (polynomial in column 0, shifted identity after it)
 * is squared to 2 and 4 zero bits, then squared once per bit of len_b, the
 * two buffers leapfrogging, applying the operator where the bit is set. */
uint32_t orc_crc32c_combine(uint32_t crc_a, uint32_t crc_b, uint64_t len_b) {
    if (len_b == 0) return crc_a;
    uint32_t a[32], b[32];
    a[0] = ORC_CRC_POLY;
    for (int i = 1; i < 32; i++) a[i] = 1u << (i - 1);
    op_square(b, a);
    op_square(a, b);
    uint32_t crc = crc_a;
    for (;;) {
        op_square(b, a);
        if (len_b & 1) crc = op_apply(b, crc);
        len_b >>= 1;
        if (!len_b) break;
        op_square(a, b);
        if (len_b & 1) crc = op_apply(a, crc);
        len_b >>= 1;
        if (!len_b) break;
    }
    return crc ^ crc_b;
}

static void put_le(uint8_t *p, uint64_t v, int bytes) {
    for (int i = 0; i < bytes; i++) p[i] = (uint8_t)(v >> (8 * i));
}

static uint64_t get_le(const uint8_t *p, int bytes) {
    uint64_t v = 0;
    for (int i = 0; i < bytes; i++) v |= (uint64_t)p[i] << (8 * i);
    return v;
}

/* block.rs:110-142: every payload becomes [4 "FQXB"][u64 len][u32 crc32c]
 * [payload], frames back to back; `terminate` appends the zero-length frame
 * that ends the block region (format.rs:318-321, the first bytes write_footer
 * emits). */
int orc_frame_blocks(const uint8_t *src, const uint64_t *off, const uint64_t *len, size_t n, int terminate,
                     uint8_t *dst, uint64_t cap, uint64_t *frame_off, uint32_t *crcs, uint64_t *total) {
    uint64_t need = terminate ? ORC_FRAME_TERM : 0;
    for (size_t i = 0; i < n; i++) need += ORC_FRAME_HEAD + len[i];
    if (total) *total = need;
    if (need > cap) return ORC_E_DST_TOO_SMALL;
    uint64_t pos = 0;
    for (size_t i = 0; i < n; i++) {
        const uint32_t c = orc_crc32c(src + off[i], len[i]);
        memcpy(dst + pos, "FQXB", 4);
        put_le(dst + pos + 4, len[i], 8);
        put_le(dst + pos + 12, c, 4);
        memcpy(dst + pos + ORC_FRAME_HEAD, src + off[i], len[i]);
        if (frame_off) frame_off[i] = pos;
        if (crcs) crcs[i] = c;
        pos += ORC_FRAME_HEAD + len[i];
    }
    if (terminate) {
        memcpy(dst + pos, "FQXB", 4);
        put_le(dst + pos + 4, 0, 8);
    }
    return ORC_OK;
}

/* block.rs:1209-1254 applied frame after frame from offset 0 of `src`:
 *   fewer than 4 bytes left             -> clean end (Ok(None))
 *   marker != "FQXB"                    -> ORC_FRAME_E_BAD_SYNC, stop
 *   fewer than 8 length bytes           -> ORC_FRAME_E_TRUNCATED, stop
 *   length 0                            -> terminator, stop (consumed)
 *   length > 2 GiB (MAX_BLOCK_PAYLOAD)  -> ORC_FRAME_E_TOO_LARGE, stop
 *   fewer than 4 CRC bytes or payload   -> ORC_FRAME_E_TRUNCATED, stop
 *   CRC-32C differs                     -> ORC_FRAME_E_CORRUPT (walk goes on)
 * A failing frame gets an entry with its status; a structural failure ends
 * the walk with `consumed` at the failing frame's start. Returns the first
 * non-OK status in frame order (the error read_block returns first). */
int orc_read_blocks(const uint8_t *src, uint64_t len, size_t max_frames, uint64_t *pay_off, uint64_t *pay_len,
                    uint32_t *crcs, int32_t *status, size_t *nframes, uint64_t *consumed, int *terminated) {
    uint64_t pos = 0;
    size_t k = 0;
    int first = ORC_OK;
    *terminated = 0;
    while (k < max_frames) {
        const uint64_t left = len - pos;
        if (left < 4) break;
        int st = ORC_OK;
        uint64_t plen = 0;
        if (memcmp(src + pos, "FQXB", 4) != 0) {
            st = ORC_FRAME_E_BAD_SYNC;
        } else if (left < 12) {
            st = ORC_FRAME_E_TRUNCATED;
        } else {
            plen = get_le(src + pos + 4, 8);
            if (plen == 0) {
                pos += ORC_FRAME_TERM;
                *terminated = 1;
                break;
            }
            if (plen > ORC_MAX_BLOCK_PAYLOAD) st = ORC_FRAME_E_TOO_LARGE;
            else if (left < ORC_FRAME_HEAD || left - ORC_FRAME_HEAD < plen) st = ORC_FRAME_E_TRUNCATED;
        }
        if (st != ORC_OK) {
            pay_off[k] = pos;
            pay_len[k] = 0;
            crcs[k] = 0;
            status[k] = st;
            if (first == ORC_OK) first = st;
            k++;
            break;
        }
        const uint32_t want = (uint32_t)get_le(src + pos + 12, 4);
        const uint32_t got = orc_crc32c(src + pos + ORC_FRAME_HEAD, plen);
        pay_off[k] = pos + ORC_FRAME_HEAD;
        pay_len[k] = plen;
        crcs[k] = got;
        status[k] = got == want ? ORC_OK : ORC_FRAME_E_CORRUPT;
        if (status[k] != ORC_OK && first == ORC_OK) first = status[k];
        k++;
        pos += ORC_FRAME_HEAD + plen;
    }
    *nframes = k;
    *consumed = pos;
    return first;
}

/* block.rs:961-980: a plain payload is [24 digests][u32 n_reads] then
 * ([u32 len][bytes]) x 3 (names, sequence, quality); each stream's location is
 * its coded bytes' absolute offset (block_offset + the 16-byte frame head +
 * offset in the payload), length and CRC-32C. A payload too short for the
 * walk is Error::Truncated. */
int orc_payload_stream_locs(const uint8_t *payload, uint64_t len, uint64_t block_offset, uint64_t loc_off[3],
                            uint32_t loc_len[3], uint32_t loc_crc[3]) {
    uint64_t p = 3 * 8 + 4;
    if (len < p) return ORC_FRAME_E_TRUNCATED;
    for (int s = 0; s < 3; s++) {
        if (len - p < 4) return ORC_FRAME_E_TRUNCATED;
        const uint32_t n = (uint32_t)get_le(payload + p, 4);
        p += 4;
        if (len - p < n) return ORC_FRAME_E_TRUNCATED;
        loc_off[s] = block_offset + ORC_FRAME_HEAD + p;
        loc_len[s] = n;
        loc_crc[s] = orc_crc32c(payload + p, n);
        p += n;
    }
    return ORC_OK;
}

/* ---- CPU baseline: CRC-32C of many spans on host threads -------------------
 * The reference checks payload CRCs on rayon workers over blocks
 * (crates/fqxv/src/container/decompress.rs:46-52 decodes blocks in parallel,
 * each read_block CRC-checked); here a thread pool takes spans off a shared
 * counter. nthreads <= 0 uses every online core. */
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <unistd.h>

typedef struct {
    const uint8_t *src;
    const uint64_t *off, *len;
    size_t n;
    uint32_t *out;
    atomic_size_t next;
} crc_job;

static void *crc_worker(void *arg) {
    crc_job *J = (crc_job *)arg;
    for (;;) {
        const size_t i = atomic_fetch_add(&J->next, 1);
        if (i >= J->n) break;
        J->out[i] = orc_crc32c(J->src + J->off[i], J->len[i]);
    }
    return NULL;
}

int orc_crc32c_batch(const uint8_t *src, const uint64_t *off, const uint64_t *len, size_t n, uint32_t *out,
                     int nthreads) {
    crc_table_init();
    if (nthreads <= 0) nthreads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nthreads < 1) nthreads = 1;
    crc_job J = {src, off, len, n, out, 0};
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nthreads);
    int started = 0;
    for (int t = 0; t < nthreads; t++)
        if (pthread_create(&th[started], NULL, crc_worker, &J) == 0) started++;
    if (started == 0) crc_worker(&J);
    for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
    free(th);
    return ORC_OK;
}
