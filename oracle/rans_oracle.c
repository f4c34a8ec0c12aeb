/*
 * Scalar restatement of crates/fqxv-rans (model.rs, scalar.rs, lib.rs).
 * TEST INFRASTRUCTURE ONLY -- see rans_oracle.h. Each function cites the
 * reference lines it follows.
 */
#include "rans_oracle.h"

#include <stdlib.h>
#include <string.h>

#define ORDER1_TABLE_BYTES (256u * 2u)

size_t orc_encode_bound(size_t n, int order) {
    if (n == 0) return 9;
    /* scalar.rs:8-20: [order][n] + tables + 32 states + <= one u16 per symbol
     * (encode_symbol emits at most one word per step, model.rs:15-16). */
    size_t tables = order == 0 ? ORDER1_TABLE_BYTES : 32 + 256 * ORDER1_TABLE_BYTES;
    return 9 + tables + 4 * ORC_N_STATES + 2 * n;
}

/* model.rs:213-264 */
void orc_normalize(const uint32_t counts[256], uint16_t freq[256]) {
    uint64_t total = 0;
    for (int s = 0; s < 256; s++) total += counts[s];
    memset(freq, 0, 256 * sizeof(uint16_t));
    if (total == 0) return;

    int64_t sum = 0;
    int max_s = 0;
    uint32_t max_f = 0;
    for (int s = 0; s < 256; s++) {
        if (counts[s] == 0) continue;
        uint32_t f = (uint32_t)(((uint64_t)counts[s] * ORC_TOTFREQ) / total);
        if (f == 0) f = 1;
        freq[s] = (uint16_t)f;
        sum += f;
        if (f > max_f) {
            max_f = f;
            max_s = s;
        }
    }
    int64_t diff = (int64_t)ORC_TOTFREQ - sum;
    while (diff != 0) {
        if (diff > 0) {
            freq[max_s] = (uint16_t)(freq[max_s] + diff);
            diff = 0;
        } else {
            int64_t take = (int64_t)freq[max_s] - 1;
            if (take < 0) take = 0;
            if (take > -diff) take = -diff;
            freq[max_s] = (uint16_t)(freq[max_s] - take);
            diff += take;
            if (diff != 0) {
                int nm = -1;
                int64_t nf = 1;
                for (int s = 0; s < 256; s++) {
                    if ((int64_t)freq[s] > nf) {
                        nf = freq[s];
                        nm = s;
                    }
                }
                if (nm < 0) return; /* unreachable: <= 256 ones sum below TOTFREQ */
                max_s = nm;
            }
        }
    }
}

/* model.rs:160-174 */
int orc_validate_freqs(const uint16_t freq[256]) {
    uint32_t acc = 0;
    for (int s = 0; s < 256; s++) {
        acc += freq[s];
        if (acc > ORC_TOTFREQ) return ORC_E_FREQ_EXCEEDS;
    }
    if (acc != ORC_TOTFREQ) return ORC_E_FREQ_SUM;
    return ORC_OK;
}

/* model.rs:52-64 */
typedef struct {
    uint64_t x_max;
    uint32_t rcp_freq, rcp_shift, bias, cmpl_freq, freq, cum;
    int use_div;
} encsym;

/* model.rs:70-119 */
static encsym encsym_new(uint32_t freq, uint32_t cum) {
    encsym e;
    memset(&e, 0, sizeof e);
    e.x_max = ((uint64_t)(ORC_RANS_L >> ORC_SCALE_BITS) << 16) * freq;
    e.freq = freq;
    e.cum = cum;
    if (freq < 2) {
        e.rcp_freq = ~0u;
        e.rcp_shift = 0;
        e.bias = cum + (1u << ORC_SCALE_BITS) - 1;
        e.cmpl_freq = (1u << ORC_SCALE_BITS) - freq;
    } else if (freq > (1u << 11)) {
        e.use_div = 1;
    } else {
        uint32_t shift = 0;
        while (freq > (1u << shift)) shift++;
        uint64_t num = 1ull << (shift + 31);
        e.rcp_freq = (uint32_t)((num + freq - 1) / freq);
        e.rcp_shift = shift - 1;
        e.bias = cum;
        e.cmpl_freq = (1u << ORC_SCALE_BITS) - freq;
    }
    return e;
}

/* model.rs:125-133 */
static inline uint32_t encsym_apply(const encsym *e, uint32_t v) {
    if (e->use_div) return ((v / e->freq) << ORC_SCALE_BITS) + (v % e->freq) + e->cum;
    uint32_t q = (uint32_t)(((uint64_t)v * e->rcp_freq) >> 32) >> e->rcp_shift;
    return v + e->bias + q * e->cmpl_freq;
}

uint32_t orc_encsym_apply(uint32_t freq, uint32_t cum, uint32_t v) {
    encsym e = encsym_new(freq, cum);
    return encsym_apply(&e, v);
}

uint32_t orc_magic_apply(uint32_t freq, uint32_t cum, uint32_t v) {
    uint32_t magic = (uint32_t)(0xffffffffull / freq);
    uint32_t q = (uint32_t)(((uint64_t)v * magic) >> 32);
    uint32_t r = v - q * freq;
    if (r >= freq) {
        q += 1;
        r -= freq;
    }
    return (q << ORC_SCALE_BITS) + r + cum;
}

/* model.rs:180-194 */
static void build_cum_slot2sym(const uint16_t freq[256], uint16_t cum[257], uint8_t *slot2sym) {
    cum[0] = 0;
    for (int s = 0; s < 256; s++) cum[s + 1] = (uint16_t)(cum[s] + freq[s]);
    if (slot2sym) {
        memset(slot2sym, 0, ORC_TOTFREQ);
        for (int s = 0; s < 256; s++)
            for (uint32_t k = cum[s]; k < cum[s + 1]; k++) slot2sym[k] = (uint8_t)s;
    }
}

/* Growable renorm word buffer (the Vec<u16> of scalar.rs:38). */
typedef struct {
    uint16_t *w;
    size_t len, cap;
} wordbuf;

static inline void wb_push(wordbuf *b, uint16_t w) { b->w[b->len++] = w; }

/* scalar.rs:120-127 */
static inline void encode_symbol(uint32_t *x, const encsym *e, wordbuf *rn) {
    uint32_t v = *x;
    while ((uint64_t)v >= e->x_max) {
        wb_push(rn, (uint16_t)(v & 0xffff));
        v >>= 16;
    }
    *x = encsym_apply(e, v);
}

static inline void put_u16(uint8_t *p, uint16_t v) {
    p[0] = (uint8_t)v;
    p[1] = (uint8_t)(v >> 8);
}
static inline void put_u32(uint8_t *p, uint32_t v) {
    for (int i = 0; i < 4; i++) p[i] = (uint8_t)(v >> (8 * i));
}
static inline void put_u64(uint8_t *p, uint64_t v) {
    for (int i = 0; i < 8; i++) p[i] = (uint8_t)(v >> (8 * i));
}

/* scalar.rs:130-140: states, then the renorm words reversed. */
static size_t finish(uint8_t *out, const uint32_t states[ORC_N_STATES], const wordbuf *rn) {
    size_t o = 0;
    for (int i = 0; i < ORC_N_STATES; i++, o += 4) put_u32(out + o, states[i]);
    for (size_t k = 0; k < rn->len; k++, o += 2) put_u16(out + o, rn->w[rn->len - 1 - k]);
    return o;
}

/* Shared by the SIMD encoders (rans_simd.c). */
size_t orc__finish(uint8_t *out, const uint32_t states[ORC_N_STATES], const uint16_t *words,
                   size_t nwords) {
    wordbuf b = {(uint16_t *)words, nwords, nwords};
    return finish(out, states, &b);
}

/* scalar.rs:29-55 */
static int encode_order0(const uint8_t *src, size_t n, uint8_t *dst, size_t *out_len) {
    uint32_t counts[256] = {0};
    for (size_t i = 0; i < n; i++) counts[src[i]]++;
    uint16_t freq[256], cum[257];
    orc_normalize(counts, freq);
    build_cum_slot2sym(freq, cum, NULL);
    encsym enc[256];
    for (int s = 0; s < 256; s++) enc[s] = encsym_new(freq[s], cum[s]);

    uint32_t states[ORC_N_STATES];
    for (int i = 0; i < ORC_N_STATES; i++) states[i] = ORC_RANS_L;
    wordbuf rn = {NULL, 0, n};
    if (n) {
        rn.w = (uint16_t *)malloc(n * sizeof(uint16_t));
        if (!rn.w) return ORC_E_INVALID_ARG;
    }
    for (size_t i = n; i-- > 0;) encode_symbol(&states[i % ORC_N_STATES], &enc[src[i]], &rn);

    size_t o = 0;
    dst[o++] = 0;
    put_u64(dst + o, (uint64_t)n);
    o += 8;
    if (n) {
        for (int s = 0; s < 256; s++, o += 2) put_u16(dst + o, freq[s]);
        o += finish(dst + o, states, &rn);
    }
    free(rn.w);
    *out_len = o;
    return ORC_OK;
}

/* scalar.rs:61-111 */
static int encode_order1(const uint8_t *src, size_t n, uint8_t *dst, size_t *out_len) {
    uint32_t *counts = (uint32_t *)calloc(256 * 256, sizeof(uint32_t));
    encsym *enc = (encsym *)malloc(256 * 256 * sizeof(encsym));
    uint16_t *freqs = (uint16_t *)calloc(256 * 256, sizeof(uint16_t));
    uint8_t present[256] = {0};
    if (!counts || !enc || !freqs) {
        free(counts);
        free(enc);
        free(freqs);
        return ORC_E_INVALID_ARG;
    }
    uint8_t prev = 0;
    for (size_t i = 0; i < n; i++) {
        counts[prev * 256 + src[i]]++;
        prev = src[i];
    }
    for (int ctx = 0; ctx < 256; ctx++) {
        int any = 0;
        for (int s = 0; s < 256; s++) any |= counts[ctx * 256 + s] != 0;
        if (!any) continue;
        present[ctx] = 1;
        uint16_t cum[257];
        orc_normalize(counts + ctx * 256, freqs + ctx * 256);
        build_cum_slot2sym(freqs + ctx * 256, cum, NULL);
        for (int s = 0; s < 256; s++) enc[ctx * 256 + s] = encsym_new(freqs[ctx * 256 + s], cum[s]);
    }

    uint32_t states[ORC_N_STATES];
    for (int i = 0; i < ORC_N_STATES; i++) states[i] = ORC_RANS_L;
    wordbuf rn = {NULL, 0, n};
    if (n) rn.w = (uint16_t *)malloc(n * sizeof(uint16_t));
    for (size_t i = n; i-- > 0;) {
        unsigned ctx = i == 0 ? 0 : src[i - 1];
        encode_symbol(&states[i % ORC_N_STATES], &enc[ctx * 256 + src[i]], &rn);
    }

    size_t o = 0;
    dst[o++] = 1;
    put_u64(dst + o, (uint64_t)n);
    o += 8;
    if (n) {
        uint8_t bitmap[32] = {0};
        for (int ctx = 0; ctx < 256; ctx++)
            if (present[ctx]) bitmap[ctx / 8] |= (uint8_t)(1u << (ctx % 8));
        memcpy(dst + o, bitmap, 32);
        o += 32;
        for (int ctx = 0; ctx < 256; ctx++) {
            if (!present[ctx]) continue;
            for (int s = 0; s < 256; s++, o += 2) put_u16(dst + o, freqs[ctx * 256 + s]);
        }
        o += finish(dst + o, states, &rn);
    }
    free(rn.w);
    free(counts);
    free(enc);
    free(freqs);
    *out_len = o;
    return ORC_OK;
}

int orc_encode(const uint8_t *src, size_t n, int order, uint8_t *dst, size_t dst_cap,
               size_t *out_len) {
    if ((order != 0 && order != 1) || !dst || !out_len || (n && !src))
        return ORC_E_INVALID_ARG;
    if (dst_cap < orc_encode_bound(n, order)) return ORC_E_DST_TOO_SMALL;
    return order == 0 ? encode_order0(src, n, dst, out_len) : encode_order1(src, n, dst, out_len);
}

/* scalar.rs:241-277 */
typedef struct {
    const uint8_t *buf;
    size_t len, pos;
} reader;

static inline int rd_take(reader *r, size_t k, const uint8_t **p) {
    if (r->len - r->pos < k || r->pos > r->len) return ORC_E_TRUNCATED;
    *p = r->buf + r->pos;
    r->pos += k;
    return ORC_OK;
}
static inline int rd_u8(reader *r, uint8_t *v) {
    const uint8_t *p;
    if (rd_take(r, 1, &p)) return ORC_E_TRUNCATED;
    *v = p[0];
    return ORC_OK;
}
static inline int rd_u16(reader *r, uint16_t *v) {
    const uint8_t *p;
    if (rd_take(r, 2, &p)) return ORC_E_TRUNCATED;
    *v = (uint16_t)(p[0] | (p[1] << 8));
    return ORC_OK;
}
static inline int rd_u32(reader *r, uint32_t *v) {
    const uint8_t *p;
    if (rd_take(r, 4, &p)) return ORC_E_TRUNCATED;
    *v = (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
    return ORC_OK;
}
static inline int rd_u64(reader *r, uint64_t *v) {
    const uint8_t *p;
    if (rd_take(r, 8, &p)) return ORC_E_TRUNCATED;
    uint64_t x = 0;
    for (int i = 7; i >= 0; i--) x = (x << 8) | p[i];
    *v = x;
    return ORC_OK;
}

/* scalar.rs:229-238 */
static inline int step_state(uint32_t *x, uint32_t f, uint32_t c, reader *r) {
    uint32_t v = f * (*x >> ORC_SCALE_BITS) + (*x & (ORC_TOTFREQ - 1)) - c;
    while (v < ORC_RANS_L) {
        uint16_t w;
        if (rd_u16(r, &w)) return ORC_E_TRUNCATED;
        v = (v << 16) | w;
    }
    *x = v;
    return ORC_OK;
}

static int read_freqs(reader *r, uint16_t freq[256]) {
    for (int s = 0; s < 256; s++)
        if (rd_u16(r, &freq[s])) return ORC_E_TRUNCATED;
    return ORC_OK;
}

/* scalar.rs:219-225 */
static int read_states(reader *r, uint32_t st[ORC_N_STATES]) {
    for (int i = 0; i < ORC_N_STATES; i++)
        if (rd_u32(r, &st[i])) return ORC_E_TRUNCATED;
    return ORC_OK;
}

/* scalar.rs:157-178 */
static int decode_order0(reader *r, size_t n, uint8_t *dst, size_t cap) {
    uint16_t freq[256], cum[257];
    uint8_t s2s[ORC_TOTFREQ];
    int e;
    if ((e = read_freqs(r, freq))) return e;
    if ((e = orc_validate_freqs(freq))) return e;
    build_cum_slot2sym(freq, cum, s2s);
    uint32_t st[ORC_N_STATES];
    if ((e = read_states(r, st))) return e;
    if (n > cap) return ORC_E_ALLOC; /* model.rs:199-205 */
    for (size_t i = 0; i < n; i++) {
        uint32_t *x = &st[i % ORC_N_STATES];
        uint8_t s = s2s[*x & (ORC_TOTFREQ - 1)];
        dst[i] = s;
        if ((e = step_state(x, freq[s], cum[s], r))) return e;
    }
    return ORC_OK;
}

/* scalar.rs:180-217 */
static int decode_order1(reader *r, size_t n, uint8_t *dst, size_t cap) {
    uint8_t bitmap[32];
    int e;
    for (int i = 0; i < 32; i++)
        if (rd_u8(r, &bitmap[i])) return ORC_E_TRUNCATED;
    uint16_t *freq = (uint16_t *)malloc(256 * 256 * sizeof(uint16_t));
    uint16_t *cum = (uint16_t *)malloc(256 * 257 * sizeof(uint16_t));
    uint8_t *s2s = (uint8_t *)malloc(256 * ORC_TOTFREQ);
    uint8_t present[256] = {0};
    e = ORC_OK;
    if (!freq || !cum || !s2s) {
        e = ORC_E_INVALID_ARG;
        goto out;
    }
    for (int ctx = 0; ctx < 256; ctx++) {
        if (!((bitmap[ctx / 8] >> (ctx % 8)) & 1)) continue;
        if ((e = read_freqs(r, freq + ctx * 256))) goto out;
        if ((e = orc_validate_freqs(freq + ctx * 256))) goto out;
        build_cum_slot2sym(freq + ctx * 256, cum + ctx * 257, s2s + ctx * ORC_TOTFREQ);
        present[ctx] = 1;
    }
    uint32_t st[ORC_N_STATES];
    if ((e = read_states(r, st))) goto out;
    if (n > cap) {
        e = ORC_E_ALLOC;
        goto out;
    }
    uint8_t prev = 0;
    for (size_t i = 0; i < n; i++) {
        unsigned ctx = i == 0 ? 0 : prev;
        if (!present[ctx]) {
            e = ORC_E_ABSENT_CONTEXT;
            goto out;
        }
        uint32_t *x = &st[i % ORC_N_STATES];
        uint8_t s = s2s[ctx * ORC_TOTFREQ + (*x & (ORC_TOTFREQ - 1))];
        dst[i] = s;
        if ((e = step_state(x, freq[ctx * 256 + s], cum[ctx * 257 + s], r))) goto out;
        prev = s;
    }
out:
    free(freq);
    free(cum);
    free(s2s);
    return e;
}

int orc_peek_output_len(const uint8_t *src, size_t len, uint64_t *n) {
    if (len < 9) return ORC_E_TRUNCATED;
    uint64_t x = 0;
    for (int i = 8; i >= 1; i--) x = (x << 8) | src[i];
    *n = x;
    return ORC_OK;
}

/* scalar.rs:143-155 */
int orc_decode(const uint8_t *src, size_t len, uint8_t *dst, size_t dst_cap, size_t *out_len) {
    if (!out_len || (len && !src)) return ORC_E_INVALID_ARG;
    reader r = {src, len, 0};
    uint8_t order;
    uint64_t n;
    if (rd_u8(&r, &order)) return ORC_E_TRUNCATED;
    if (rd_u64(&r, &n)) return ORC_E_TRUNCATED;
    *out_len = 0;
    if (n == 0) return ORC_OK;
    int e;
    if (order == 0)
        e = decode_order0(&r, (size_t)n, dst, dst_cap);
    else if (order == 1)
        e = decode_order1(&r, (size_t)n, dst, dst_cap);
    else
        return ORC_E_UNKNOWN_ORDER;
    if (e == ORC_OK) *out_len = (size_t)n;
    return e;
}

/* lib.rs:226-231 */
int orc_decode_bounded(const uint8_t *src, size_t len, size_t max_len, uint8_t *dst,
                       size_t dst_cap, size_t *out_len) {
    uint64_t n;
    if (orc_peek_output_len(src, len, &n) == ORC_OK && n > (uint64_t)max_len) return ORC_E_BOUND;
    return orc_decode(src, len, dst, dst_cap, out_len);
}

/* lib.rs:111-127 */
int orc_encode_dispatch(const uint8_t *src, size_t n, int order, uint8_t *dst, size_t dst_cap,
                        size_t *out_len) {
    int lvl = orc_simd_level();
    if (order == 0 && lvl > 0) return orc_encode_o0_simd(lvl, src, n, dst, dst_cap, out_len);
    return orc_encode(src, n, order, dst, dst_cap, out_len);
}

/* lib.rs:186-200 */
int orc_decode_dispatch(const uint8_t *src, size_t len, uint8_t *dst, size_t dst_cap,
                        size_t *out_len) {
    int lvl = orc_simd_level();
    if (len >= 1 && src[0] == 0 && lvl > 0) return orc_decode_o0_simd(lvl, src, len, dst, dst_cap, out_len);
    return orc_decode(src, len, dst, dst_cap, out_len);
}

/* model.rs:313-365: the reciprocal/division split (and the SIMD magic form)
 * must equal `(v / f) << 12 + v % f + c` for every frequency over its renorm
 * interval [x_max >> 16, x_max), endpoints and the 2^31 window included.
 * Returns the number of mismatches. */
size_t orc_check_apply_sweep(void) {
    size_t bad = 0;
    for (uint32_t freq = 1; freq <= ORC_TOTFREQ; freq++) {
        uint32_t cum = ORC_TOTFREQ - freq < 100 ? ORC_TOTFREQ - freq : 100;
        uint64_t x_max = (uint64_t)freq << 20;
        uint64_t lo = (x_max >> 16) > 1 ? (x_max >> 16) : 1;
        uint64_t step = (x_max - lo) / 512 > 1 ? (x_max - lo) / 512 : 1;
#define CHECK(vv)                                                                  \
    do {                                                                           \
        uint32_t v_ = (uint32_t)(vv);                                              \
        uint32_t want = ((v_ / freq) << ORC_SCALE_BITS) + (v_ % freq) + cum;        \
        bad += orc_encsym_apply(freq, cum, v_) != want;                            \
        bad += orc_magic_apply(freq, cum, v_) != want;                             \
    } while (0)
        CHECK(lo);
        CHECK(x_max - 1);
        if (x_max > (1ull << 31)) {
            CHECK(1u << 31);
            CHECK((1u << 31) + 1);
        }
        for (uint64_t v = lo; v < x_max; v += step) CHECK(v);
    }
    const uint32_t edge[5] = {1u << 11, (1u << 11) + 1, 3000, 4095, ORC_TOTFREQ};
    for (int k = 0; k < 5; k++) {
        uint32_t freq = edge[k], cum = 7;
        uint64_t x_max = (uint64_t)freq << 20;
        for (uint64_t d = 0; d < 200000; d++) {
            uint64_t vs[2] = {(1ull << 31) + d, (1ull << 31) - d};
            for (int j = 0; j < 2; j++) {
                if (vs[j] >= x_max || vs[j] < (x_max >> 16)) continue;
                CHECK(vs[j]);
            }
        }
    }
#undef CHECK
    return bad;
}
