/*
 * CPU oracle of the extended stream format (a new format tag) -- TEST
 * INFRASTRUCTURE ONLY, like the rest of oracle/.
 *
 * PARITY UNPINNED: the reference crate writes one format only, 32
 * interleaved states with a flag-less `[u8 order][u64 n]` header
 * (crates/fqxv-rans/src/model.rs:19, scalar.rs:8-20), and has no raw path
 * (docs/design/testing.md:141-143). The 4-way interleave and the
 * STRIPE / RLE / PACK / CAT transforms below have no reference
 * implementation; this file defines them and is the checker of the GPU
 * implementation. Their 32-way cores are reference streams, written by the
 * restatement of scalar.rs (orc_encode), so those bytes stay pinned.
 *
 * Extended stream:  [u8 0x80 | flags][u64 n] body       (n == 0: no body)
 *   flags  ORC_X_ORDER1  cores use the order-1 model (else order-0)
 *          ORC_X_N4      cores use 4 interleaved states (else 32)
 *          ORC_X_STRIPE  body = [4 x u64 length] + 4 complete nested streams;
 *                        stream j codes bytes j, j + 4, j + 8, ...; any other
 *                        flag is then ignored at this level
 *          ORC_X_PACK    [u8 nsym][nsym symbols, ascending]; symbol k becomes
 *                        code k, codes packed LSB first, 0 bits (nsym 1),
 *                        1 bit (<= 2), 2 bits (<= 4) or 4 bits (<= 16) each
 *          ORC_X_RLE     [u8 nrun][nrun run symbols, ascending][u64 nlit]
 *                        [u64 nrb]; every maximal run of a run symbol becomes
 *                        one literal plus (length - 1) as a LEB128 varint in
 *                        the run-byte array; other symbols stay literals
 *          ORC_X_CAT     cores are the arrays' raw bytes
 *   then one core per array: the packed (or plain) bytes, or the literal and
 *   the run-byte arrays for RLE. A core is [u64 byte length][stream]; the
 *   stream is a reference stream (32 states) or, with ORC_X_N4, the same
 *   layout with tag 2 | order and 4 states. CAT cores are the raw bytes
 *   (their length is known from the header).
 */
#include "rans_oracle.h"

#include <stdlib.h>
#include <string.h>

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
static inline uint64_t get_u64(const uint8_t *p) {
    uint64_t v = 0;
    for (int i = 7; i >= 0; i--) v = (v << 8) | p[i];
    return v;
}
static inline uint32_t get_u32(const uint8_t *p) {
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

/* ---- 4-way cores ----------------------------------------------------------
 * The reference's arithmetic (model.rs:70-133, scalar.rs:120-127, 143-238)
 * with 4 states: state i % 4 codes position i. The encode map is computed by
 * exact division; any exact method gives the same state. */

#define N4 4

size_t orc_core_bound(size_t n, int order, int nstates) {
    if (n == 0) return 9;
    size_t tables = order == 0 ? 512 : 32 + 256 * 512;
    return 9 + tables + 4 * (size_t)nstates + 2 * n;
}

static void cum_of(const uint16_t f[256], uint32_t cum[257]) {
    cum[0] = 0;
    for (int s = 0; s < 256; s++) cum[s + 1] = cum[s] + f[s];
}

static inline void n4_put(uint32_t *x, uint32_t f, uint32_t c, uint16_t *words, size_t *nw) {
    uint32_t v = *x;
    const uint64_t xmax = (uint64_t)f << 20;
    while ((uint64_t)v >= xmax) {
        words[(*nw)++] = (uint16_t)(v & 0xffff);
        v >>= 16;
    }
    *x = ((v / f) << ORC_SCALE_BITS) + (v % f) + c;
}

static int core_encode_n4(const uint8_t *src, size_t n, int order, uint8_t *dst, size_t *out_len) {
    size_t o = 0;
    dst[o++] = (uint8_t)(2 | order);
    put_u64(dst + o, (uint64_t)n);
    o += 8;
    if (n == 0) {
        *out_len = o;
        return ORC_OK;
    }
    uint16_t *words = (uint16_t *)malloc(n * sizeof(uint16_t));
    uint32_t *counts = (uint32_t *)calloc(order ? 65536 : 256, sizeof(uint32_t));
    uint16_t *freqs = (uint16_t *)calloc(order ? 65536 : 256, sizeof(uint16_t));
    uint32_t *cums = (uint32_t *)calloc(order ? 256 * 257 : 257, sizeof(uint32_t));
    if (!words || !counts || !freqs || !cums) {
        free(words), free(counts), free(freqs), free(cums);
        return ORC_E_INVALID_ARG;
    }
    uint8_t present[256] = {0};
    if (order == 0) {
        for (size_t i = 0; i < n; i++) counts[src[i]]++;
        orc_normalize(counts, freqs);
        cum_of(freqs, cums);
    } else {
        uint8_t prev = 0;
        for (size_t i = 0; i < n; i++) {
            counts[prev * 256 + src[i]]++;
            prev = src[i];
        }
        for (int c = 0; c < 256; c++) {
            int any = 0;
            for (int s = 0; s < 256; s++) any |= counts[c * 256 + s] != 0;
            if (!any) continue;
            present[c] = 1;
            orc_normalize(counts + c * 256, freqs + c * 256);
            cum_of(freqs + c * 256, cums + c * 257);
        }
    }
    uint32_t st[N4];
    for (int i = 0; i < N4; i++) st[i] = ORC_RANS_L;
    size_t nw = 0;
    for (size_t i = n; i-- > 0;) {
        const unsigned s = src[i];
        const unsigned c = order ? (i ? src[i - 1] : 0u) : 0u;
        const uint32_t f = freqs[c * 256 * order + s];
        const uint32_t cu = cums[c * 257 * order + s];
        n4_put(&st[i % N4], f, cu, words, &nw);
    }
    if (order == 0) {
        for (int s = 0; s < 256; s++, o += 2) put_u16(dst + o, freqs[s]);
    } else {
        uint8_t bitmap[32] = {0};
        for (int c = 0; c < 256; c++)
            if (present[c]) bitmap[c / 8] |= (uint8_t)(1u << (c % 8));
        memcpy(dst + o, bitmap, 32);
        o += 32;
        for (int c = 0; c < 256; c++) {
            if (!present[c]) continue;
            for (int s = 0; s < 256; s++, o += 2) put_u16(dst + o, freqs[c * 256 + s]);
        }
    }
    for (int i = 0; i < N4; i++, o += 4) put_u32(dst + o, st[i]);
    for (size_t k = 0; k < nw; k++, o += 2) put_u16(dst + o, words[nw - 1 - k]);
    free(words), free(counts), free(freqs), free(cums);
    *out_len = o;
    return ORC_OK;
}

/* A table of 256 u16 read at p (in bounds): validate (model.rs:160-174), cum,
 * slot -> symbol. */
static int n4_table(const uint8_t *p, uint16_t f[256], uint32_t cum[257], uint8_t *slot2sym) {
    for (int s = 0; s < 256; s++) f[s] = (uint16_t)(p[2 * s] | (p[2 * s + 1] << 8));
    int st = orc_validate_freqs(f);
    if (st) return st;
    cum_of(f, cum);
    for (int s = 0; s < 256; s++)
        for (uint32_t k = cum[s]; k < cum[s + 1]; k++) slot2sym[k] = (uint8_t)s;
    return ORC_OK;
}

static int core_decode_n4(const uint8_t *src, size_t len, uint8_t *dst, size_t cap, size_t *out_len) {
    if (len < 9) return ORC_E_TRUNCATED;
    const int order = src[0] & 1;
    const uint64_t n = get_u64(src + 1);
    if (n == 0) {
        *out_len = 0;
        return ORC_OK;
    }
    size_t pos = 9;
    int ntab = 1;
    uint16_t ctxidx[256]; /* present context -> table index; 0xffff: absent */
    for (int c = 0; c < 256; c++) ctxidx[c] = 0xffff;
    if (order) {
        if (len < pos + 32) return ORC_E_TRUNCATED;
        ntab = 0;
        for (int c = 0; c < 256; c++)
            if ((src[pos + c / 8] >> (c % 8)) & 1) ctxidx[c] = (uint16_t)ntab++;
        pos += 32;
    }
    const int alloc = ntab ? ntab : 1;
    uint16_t *f = (uint16_t *)malloc((size_t)alloc * 256 * sizeof(uint16_t));
    uint32_t *cum = (uint32_t *)malloc((size_t)alloc * 257 * sizeof(uint32_t));
    uint8_t *s2s = (uint8_t *)malloc((size_t)alloc * 4096);
    int st = ORC_OK;
    if (!f || !cum || !s2s) st = ORC_E_INVALID_ARG;
    for (int t = 0; t < ntab && st == ORC_OK; t++) {
        if (len < pos + 512) {
            st = ORC_E_TRUNCATED;
            break;
        }
        st = n4_table(src + pos, f + t * 256, cum + t * 257, s2s + (size_t)t * 4096);
        pos += 512;
    }
    uint32_t x[N4];
    if (st == ORC_OK && len < pos + 4 * N4) st = ORC_E_TRUNCATED;
    if (st == ORC_OK && n > cap) st = ORC_E_ALLOC;
    if (st == ORC_OK) {
        for (int i = 0; i < N4; i++) x[i] = get_u32(src + pos + 4 * i);
        pos += 4 * N4;
        unsigned ctx = 0;
        for (uint64_t i = 0; i < n && st == ORC_OK; i++) {
            uint32_t *xs = &x[i % N4];
            unsigned t = 0;
            if (order) {
                if (ctxidx[ctx] == 0xffff) {
                    st = ORC_E_ABSENT_CONTEXT;
                    break;
                }
                t = ctxidx[ctx];
            }
            const uint32_t slot = *xs & (ORC_TOTFREQ - 1);
            const unsigned s = s2s[(size_t)t * 4096 + slot];
            uint32_t v = f[t * 256 + s] * (*xs >> ORC_SCALE_BITS) + slot - cum[t * 257 + s];
            while (v < ORC_RANS_L) {
                if (len < pos + 2) {
                    st = ORC_E_TRUNCATED;
                    break;
                }
                v = (v << 16) | (uint32_t)(src[pos] | (src[pos + 1] << 8));
                pos += 2;
            }
            *xs = v;
            dst[i] = (uint8_t)s;
            ctx = s;
        }
    }
    free(f), free(cum), free(s2s);
    if (st == ORC_OK) *out_len = (size_t)n;
    return st;
}

int orc_core_encode(const uint8_t *src, size_t n, int order, int nstates, uint8_t *dst, size_t *out_len) {
    if (nstates == ORC_N_STATES) return orc_encode(src, n, order, dst, orc_encode_bound(n, order), out_len);
    if (nstates != N4 || (order != 0 && order != 1)) return ORC_E_INVALID_ARG;
    return core_encode_n4(src, n, order, dst, out_len);
}

int orc_core_decode(const uint8_t *src, size_t len, uint8_t *dst, size_t cap, size_t *out_len) {
    if (len >= 1 && (src[0] == 2 || src[0] == 3)) return core_decode_n4(src, len, dst, cap, out_len);
    return orc_decode(src, len, dst, cap, out_len);
}

/* ---- transforms ------------------------------------------------------------ */

static int pack_bits(int nsym) { return nsym <= 1 ? 0 : nsym <= 2 ? 1 : nsym <= 4 ? 2 : 4; }

/* Symbols of src in ascending order; returns their count. */
static int symbol_set(const uint8_t *src, size_t n, uint8_t syms[256]) {
    uint8_t seen[256] = {0};
    for (size_t i = 0; i < n; i++) seen[src[i]] = 1;
    int k = 0;
    for (int s = 0; s < 256; s++)
        if (seen[s]) syms[k++] = (uint8_t)s;
    return k;
}

/* Run symbols of src: those whose occurrences exceed twice their runs
 * (average run length above 2), ascending. */
static int run_symbols(const uint8_t *src, size_t n, uint8_t syms[256], uint8_t isrun[256]) {
    uint64_t occ[256] = {0}, runs[256] = {0};
    for (size_t i = 0; i < n; i++) {
        occ[src[i]]++;
        if (i == 0 || src[i] != src[i - 1]) runs[src[i]]++;
    }
    int k = 0;
    memset(isrun, 0, 256);
    for (int s = 0; s < 256; s++)
        if (occ[s] > 2 * runs[s]) {
            syms[k++] = (uint8_t)s;
            isrun[s] = 1;
        }
    return k;
}

static size_t varint_put(uint8_t *p, uint64_t v) {
    size_t k = 0;
    while (v >= 0x80) {
        p[k++] = (uint8_t)(v | 0x80);
        v >>= 7;
    }
    p[k++] = (uint8_t)v;
    return k;
}

/* Without STRIPE: header, PACK and RLE metadata, and up to two cores. Each of
 * RLE's two arrays holds at most n bytes (a literal stands for at least one
 * position, and a run of L positions gets a varint of at most L bytes), so
 * two cores of at most n symbols each, or 2n raw bytes, cover them. */
static size_t flat_bound(size_t n) {
    if (n == 0) return 9;
    return 9 + 1 + 256 + 1 + 256 + 16 + 2 * (8 + orc_core_bound(n, 1, ORC_N_STATES)) + 2 * n;
}

static size_t nested_best_bound(size_t n) {
    const size_t r = orc_encode_bound(n, 1);
    const size_t f = flat_bound(n);
    return r > f ? r : f;
}

size_t orc_x_encode_bound(size_t n, int flags) {
    if (n == 0) return 9;
    if (flags & ORC_X_STRIPE) {
        size_t b = 9 + 32;
        for (int j = 0; j < 4; j++) b += nested_best_bound((n + 3 - j) / 4);
        return b;
    }
    return flat_bound(n);
}

int orc_x_encode_best_nested(const uint8_t *src, size_t n, uint8_t *dst, size_t *out_len, int *cand);

/* One core of array a[0, m): raw (CAT) or [u64 len][stream]. */
static int put_core(const uint8_t *a, size_t m, int flags, uint8_t *dst, size_t *o) {
    if (flags & ORC_X_CAT) {
        if (m) memcpy(dst + *o, a, m);
        *o += m;
        return ORC_OK;
    }
    size_t len = 0;
    const int st = orc_core_encode(a, m, flags & ORC_X_ORDER1 ? 1 : 0, flags & ORC_X_N4 ? N4 : ORC_N_STATES,
                                   dst + *o + 8, &len);
    if (st) return st;
    put_u64(dst + *o, (uint64_t)len);
    *o += 8 + len;
    return ORC_OK;
}

int orc_x_encode(const uint8_t *src, size_t n, int flags, uint8_t *dst, size_t dst_cap, size_t *out_len) {
    if (!dst || !out_len || (n && !src) || (flags & ~ORC_X_ALL)) return ORC_E_INVALID_ARG;
    if (dst_cap < orc_x_encode_bound(n, flags)) return ORC_E_DST_TOO_SMALL;
    size_t o = 0;
    dst[o++] = (uint8_t)(0x80 | flags);
    put_u64(dst + o, (uint64_t)n);
    o += 8;
    if (n == 0) {
        *out_len = o;
        return ORC_OK;
    }
    int st = ORC_OK;
    if (flags & ORC_X_STRIPE) {
        const size_t lens_at = o;
        o += 32;
        uint8_t *plane = (uint8_t *)malloc((n + 3) / 4);
        if (!plane) return ORC_E_INVALID_ARG;
        for (int j = 0; j < 4 && st == ORC_OK; j++) {
            const size_t nj = (n + 3 - j) / 4;
            for (size_t i = 0; i < nj; i++) plane[i] = src[4 * i + j];
            size_t len = 0;
            int fl = 0;
            st = orc_x_encode_best_nested(plane, nj, dst + o, &len, &fl);
            put_u64(dst + lens_at + 8 * j, (uint64_t)len);
            o += len;
        }
        free(plane);
        *out_len = o;
        return st;
    }
    const uint8_t *a = src;
    size_t m = n;
    uint8_t *packed = NULL, *lits = NULL, *rb = NULL;
    if (flags & ORC_X_PACK) {
        uint8_t syms[256];
        const int nsym = symbol_set(src, n, syms);
        if (nsym > 16) return ORC_E_INVALID_ARG;
        const int bits = pack_bits(nsym);
        uint8_t code[256] = {0};
        for (int k = 0; k < nsym; k++) code[syms[k]] = (uint8_t)k;
        dst[o++] = (uint8_t)nsym;
        memcpy(dst + o, syms, (size_t)nsym);
        o += (size_t)nsym;
        m = (n * (size_t)bits + 7) / 8;
        packed = (uint8_t *)calloc(m ? m : 1, 1);
        if (!packed) return ORC_E_INVALID_ARG;
        if (bits) {
            const size_t per = 8 / (size_t)bits;
            for (size_t i = 0; i < n; i++)
                packed[i / per] |= (uint8_t)(code[src[i]] << ((i % per) * (size_t)bits));
        }
        a = packed;
    }
    if (flags & ORC_X_RLE) {
        uint8_t syms[256], isrun[256];
        const int nrun = run_symbols(a, m, syms, isrun);
        dst[o++] = (uint8_t)nrun;
        memcpy(dst + o, syms, (size_t)nrun);
        o += (size_t)nrun;
        lits = (uint8_t *)malloc(m ? m : 1);
        rb = (uint8_t *)malloc(m ? m : 1);
        if (!lits || !rb) {
            free(packed), free(lits), free(rb);
            return ORC_E_INVALID_ARG;
        }
        size_t nl = 0, nb = 0;
        for (size_t i = 0; i < m;) {
            size_t j = i + 1;
            while (j < m && a[j] == a[i]) j++;
            if (isrun[a[i]]) {
                lits[nl++] = a[i];
                nb += varint_put(rb + nb, (uint64_t)(j - i - 1));
            } else {
                for (size_t k = i; k < j; k++) lits[nl++] = a[i];
            }
            i = j;
        }
        put_u64(dst + o, (uint64_t)nl);
        put_u64(dst + o + 8, (uint64_t)nb);
        o += 16;
        st = put_core(lits, nl, flags, dst, &o);
        if (st == ORC_OK) st = put_core(rb, nb, flags, dst, &o);
    } else {
        st = put_core(a, m, flags, dst, &o);
    }
    free(packed), free(lits), free(rb);
    *out_len = o;
    return st;
}

/* Core of m bytes at src[*pos, len) into out (cap m). */
static int get_core(const uint8_t *src, size_t len, size_t *pos, int flags, uint8_t *out, size_t m) {
    if (flags & ORC_X_CAT) {
        if (len - *pos < m) return ORC_E_TRUNCATED;
        if (m) memcpy(out, src + *pos, m);
        *pos += m;
        return ORC_OK;
    }
    if (len - *pos < 8) return ORC_E_TRUNCATED;
    const uint64_t cl = get_u64(src + *pos);
    *pos += 8;
    if (cl > len - *pos) return ORC_E_TRUNCATED;
    const uint8_t *c = src + *pos;
    /* the core's order and width must be the ones the flags declare */
    const int want = (flags & ORC_X_N4 ? 2 : 0) | (flags & ORC_X_ORDER1 ? 1 : 0);
    if (cl < 9 || c[0] != want) return cl < 9 ? ORC_E_TRUNCATED : ORC_E_X_MALFORMED;
    if (get_u64(c + 1) != (uint64_t)m) return ORC_E_X_MALFORMED;
    size_t got = 0;
    const int st = orc_core_decode(c, (size_t)cl, out, m, &got);
    *pos += (size_t)cl;
    return st;
}

int orc_x_decode(const uint8_t *src, size_t len, uint8_t *dst, size_t dst_cap, size_t *out_len) {
    if (!src || !dst || !out_len) return ORC_E_INVALID_ARG;
    if (len < 9) return ORC_E_TRUNCATED;
    if (src[0] < 0x80) return orc_decode(src, len, dst, dst_cap, out_len);
    const int flags = src[0] & 0x7f;
    const uint64_t n = get_u64(src + 1);
    if (n == 0) {
        *out_len = 0;
        return ORC_OK;
    }
    if (flags & ~ORC_X_ALL) return ORC_E_UNKNOWN_ORDER;
    if (n > dst_cap) return ORC_E_ALLOC;
    size_t pos = 9;
    int st = ORC_OK;
    if (flags & ORC_X_STRIPE) {
        if (len < pos + 32) return ORC_E_TRUNCATED;
        uint64_t lens[4];
        for (int j = 0; j < 4; j++) lens[j] = get_u64(src + pos + 8 * j);
        pos += 32;
        uint8_t *plane = (uint8_t *)malloc((size_t)(n + 3) / 4);
        if (!plane) return ORC_E_INVALID_ARG;
        for (int j = 0; j < 4 && st == ORC_OK; j++) {
            const size_t nj = (size_t)(n + 3 - j) / 4;
            if (lens[j] > len - pos) {
                st = ORC_E_TRUNCATED;
                break;
            }
            size_t got = 0;
            st = orc_x_decode(src + pos, (size_t)lens[j], plane, nj, &got);
            if (st == ORC_OK && got != nj) st = ORC_E_X_MALFORMED;
            for (size_t i = 0; st == ORC_OK && i < nj; i++) dst[4 * i + j] = plane[i];
            pos += (size_t)lens[j];
        }
        free(plane);
        if (st == ORC_OK) *out_len = (size_t)n;
        return st;
    }
    uint8_t syms[256] = {0};
    int nsym = 0, bits = 8;
    size_t m = (size_t)n;
    if (flags & ORC_X_PACK) {
        if (len < pos + 1) return ORC_E_TRUNCATED;
        nsym = src[pos++];
        if (nsym < 1 || nsym > 16) return ORC_E_X_MALFORMED;
        if (len < pos + (size_t)nsym) return ORC_E_TRUNCATED;
        memcpy(syms, src + pos, (size_t)nsym);
        pos += (size_t)nsym;
        bits = pack_bits(nsym);
        m = ((size_t)n * (size_t)bits + 7) / 8;
    }
    uint8_t *a = (uint8_t *)malloc(m ? m : 1);
    if (!a) return ORC_E_INVALID_ARG;
    if (flags & ORC_X_RLE) {
        uint8_t isrun[256] = {0};
        if (len < pos + 1) st = ORC_E_TRUNCATED;
        int nrun = st ? 0 : src[pos++];
        if (st == ORC_OK && len < pos + (size_t)nrun + 16) st = ORC_E_TRUNCATED;
        uint64_t nl = 0, nb = 0;
        if (st == ORC_OK) {
            for (int k = 0; k < nrun; k++) isrun[src[pos + k]] = 1;
            pos += (size_t)nrun;
            nl = get_u64(src + pos);
            nb = get_u64(src + pos + 8);
            pos += 16;
            if (nl > m || nb > m) st = ORC_E_X_MALFORMED;
        }
        uint8_t *lits = NULL, *rb = NULL;
        if (st == ORC_OK) {
            lits = (uint8_t *)malloc(nl ? (size_t)nl : 1);
            rb = (uint8_t *)malloc(nb ? (size_t)nb : 1);
            if (!lits || !rb) st = ORC_E_INVALID_ARG;
        }
        if (st == ORC_OK) st = get_core(src, len, &pos, flags, lits, (size_t)nl);
        if (st == ORC_OK) st = get_core(src, len, &pos, flags, rb, (size_t)nb);
        size_t w = 0, r = 0;
        for (uint64_t k = 0; st == ORC_OK && k < nl; k++) {
            uint64_t run = 1;
            if (isrun[lits[k]]) {
                uint64_t v = 0;
                int sh = 0;
                for (;;) {
                    if (r >= nb || sh > 56) {
                        st = ORC_E_X_MALFORMED;
                        break;
                    }
                    const uint8_t b = rb[r++];
                    v |= (uint64_t)(b & 0x7f) << sh;
                    sh += 7;
                    if (!(b & 0x80)) break;
                }
                run = v + 1;
            }
            if (st || run > m - w) {
                st = ORC_E_X_MALFORMED;
                break;
            }
            memset(a + w, lits[k], (size_t)run);
            w += (size_t)run;
        }
        if (st == ORC_OK && (w != m || r != nb)) st = ORC_E_X_MALFORMED;
        free(lits), free(rb);
    } else {
        st = get_core(src, len, &pos, flags, a, m);
    }
    if (st == ORC_OK) {
        if (flags & ORC_X_PACK) {
            if (bits == 0) {
                memset(dst, syms[0], (size_t)n);
            } else {
                const size_t per = 8 / (size_t)bits;
                const unsigned mask = (1u << bits) - 1u;
                for (size_t i = 0; i < (size_t)n; i++) {
                    const unsigned c = (a[i / per] >> ((i % per) * (size_t)bits)) & mask;
                    if ((int)c >= nsym) {
                        st = ORC_E_X_MALFORMED;
                        break;
                    }
                    dst[i] = syms[c];
                }
            }
        } else {
            memcpy(dst, a, (size_t)n);
        }
    }
    free(a);
    if (st == ORC_OK) *out_len = (size_t)n;
    return st;
}

/* ---- selection -------------------------------------------------------------
 * Candidates in a fixed order; the smallest stream wins and ties keep the
 * earlier candidate:
 *   0, 1  reference streams, order 0 and 1 (the untagged format)
 *   2, 3  PACK, order 0 / 1           (alphabets of at most 16 symbols)
 *   4, 5  RLE, order 0 / 1
 *   6, 7  PACK + RLE, order 0 / 1     (alphabets of at most 16 symbols)
 *   8     STRIPE, each plane by this same selection without STRIPE
 *   9     CAT
 * Nested STRIPE planes use candidates 0-7 and 9. */
static const int kCand[10] = {-1, -2, ORC_X_PACK, ORC_X_PACK | ORC_X_ORDER1, ORC_X_RLE, ORC_X_RLE | ORC_X_ORDER1,
                              ORC_X_PACK | ORC_X_RLE, ORC_X_PACK | ORC_X_RLE | ORC_X_ORDER1, ORC_X_STRIPE,
                              ORC_X_CAT};

static int encode_candidate(const uint8_t *src, size_t n, int c, uint8_t *dst, size_t *len) {
    if (kCand[c] == -1) return orc_encode(src, n, 0, dst, orc_encode_bound(n, 0), len);
    if (kCand[c] == -2) return orc_encode(src, n, 1, dst, orc_encode_bound(n, 1), len);
    return orc_x_encode(src, n, kCand[c], dst, orc_x_encode_bound(n, kCand[c]), len);
}

static int best_of(const uint8_t *src, size_t n, int nested, uint8_t *dst, size_t *out_len, int *cand_out) {
    uint8_t syms[256];
    const int nsym = symbol_set(src, n, syms);
    uint8_t *tmp = (uint8_t *)malloc(orc_x_best_bound(n));
    if (!tmp) return ORC_E_INVALID_ARG;
    size_t best = (size_t)-1;
    int bc = -1;
    for (int c = 0; c < 10; c++) {
        if (nested && c == 8) continue;
        if (kCand[c] > 0 && (kCand[c] & ORC_X_PACK) && nsym > 16) continue;
        if (c == 8 && n < 4) continue;
        size_t len = 0;
        const int st = encode_candidate(src, n, c, tmp, &len);
        if (st) {
            free(tmp);
            return st;
        }
        if (len < best) {
            best = len;
            bc = c;
            memcpy(dst, tmp, len);
        }
    }
    free(tmp);
    *out_len = best;
    if (cand_out) *cand_out = bc;
    return ORC_OK;
}

int orc_x_encode_best_nested(const uint8_t *src, size_t n, uint8_t *dst, size_t *out_len, int *cand) {
    return best_of(src, n, 1, dst, out_len, cand);
}

size_t orc_x_best_bound(size_t n) {
    const size_t a = nested_best_bound(n), b = orc_x_encode_bound(n, ORC_X_STRIPE);
    return a > b ? a : b;
}

int orc_x_encode_best(const uint8_t *src, size_t n, uint8_t *dst, size_t dst_cap, size_t *out_len, int *cand) {
    if (!dst || !out_len || (n && !src)) return ORC_E_INVALID_ARG;
    if (dst_cap < orc_x_best_bound(n)) return ORC_E_DST_TOO_SMALL;
    return best_of(src, n, 0, dst, out_len, cand);
}

/* ---- block-parallel batch over all host cores (the CPU check of the GPU's
 * batches): flags a transform combination, or 0x40 for the selection. ---- */
#include <pthread.h>
#include <stdatomic.h>
#include <unistd.h>

typedef struct {
    const uint8_t *src;
    const uint64_t *src_off, *src_len;
    size_t nblocks;
    int flags, decode;
    uint8_t *dst;
    const uint64_t *dst_off, *dst_cap;
    uint64_t *out_len;
    int32_t *status, *choice;
    atomic_size_t next;
} x_job;

static void *x_worker(void *arg) {
    x_job *J = (x_job *)arg;
    for (;;) {
        const size_t i = atomic_fetch_add(&J->next, 1);
        if (i >= J->nblocks) break;
        const uint8_t *s = J->src + J->src_off[i];
        uint8_t *d = J->dst + J->dst_off[i];
        size_t ol = 0;
        int st, c = J->flags;
        if (J->decode)
            st = orc_x_decode(s, J->src_len[i], d, J->dst_cap[i], &ol);
        else if (J->flags == 0x40)
            st = orc_x_encode_best(s, J->src_len[i], d, J->dst_cap[i], &ol, &c);
        else
            st = orc_x_encode(s, J->src_len[i], J->flags, d, J->dst_cap[i], &ol);
        J->out_len[i] = ol;
        J->status[i] = st;
        if (J->choice) J->choice[i] = c;
    }
    return NULL;
}

int orc_x_batch(const uint8_t *src, const uint64_t *src_off, const uint64_t *src_len, size_t nblocks, int flags,
                int decode, uint8_t *dst, const uint64_t *dst_off, const uint64_t *dst_cap, uint64_t *out_len,
                int32_t *status, int32_t *choice, int nthreads) {
    x_job J = {src, src_off, src_len, nblocks, flags, decode, dst, dst_off, dst_cap, out_len, status, choice};
    atomic_init(&J.next, 0);
    if (nthreads <= 0) nthreads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nthreads < 1) nthreads = 1;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nthreads);
    int started = 0;
    for (int t = 1; t < nthreads && th; t++)
        if (pthread_create(&th[started], NULL, x_worker, &J) == 0) started++;
    x_worker(&J);
    for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
    free(th);
    for (size_t i = 0; i < nblocks; i++)
        if (status[i]) return status[i];
    return ORC_OK;
}
