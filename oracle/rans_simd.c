/*
 * Restatement of the reference's order-0 SIMD backends
 * (crates/fqxv-rans/src/avx2.rs, avx512.rs) plus a block-parallel batch
 * driver -- TEST INFRASTRUCTURE ONLY (the timed CPU baseline and a
 * cross-check that the SIMD encoders are byte-identical to scalar).
 */
#include <immintrin.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "rans_oracle.h"

size_t orc__finish(uint8_t *out, const uint32_t states[ORC_N_STATES], const uint16_t *words,
                   size_t nwords);

int orc_simd_level(void) {
    static int lvl = -1;
    if (lvl < 0) {
        __builtin_cpu_init();
        lvl = __builtin_cpu_supports("avx512f") ? 2 : __builtin_cpu_supports("avx2") ? 1 : 0;
    }
    return lvl;
}

/* ---------------- shared model pieces (model.rs / avx2.rs) ---------------- */

typedef struct {
    uint16_t freq[256];
    uint16_t cum[257];
    uint8_t slot2sym[ORC_TOTFREQ];
} model0;

static void model_from_freqs(model0 *m) {
    m->cum[0] = 0;
    for (int s = 0; s < 256; s++) m->cum[s + 1] = (uint16_t)(m->cum[s] + m->freq[s]);
    for (int s = 0; s < 256; s++)
        for (uint32_t k = m->cum[s]; k < m->cum[s + 1]; k++) m->slot2sym[k] = (uint8_t)s;
}

/* avx2.rs:37-54: ((freq-1) << 20) | (offset << 8) | sym per slot. */
static void slot_table(const model0 *m, int32_t *packed) {
    for (uint32_t slot = 0; slot < ORC_TOTFREQ; slot++) {
        uint8_t s = m->slot2sym[slot];
        uint32_t f = m->freq[s], c = m->cum[s];
        packed[slot] = (int32_t)(((f - 1) << 20) | ((slot - c) << 8) | s);
    }
}

/* avx2.rs:245-264 */
static void enc_tables(const model0 *m, int32_t *magic, int32_t *fc) {
    for (int s = 0; s < 256; s++) {
        uint32_t f = m->freq[s];
        magic[s] = 0;
        fc[s] = 0;
        if (!f) continue;
        magic[s] = (int32_t)(uint32_t)(0xffffffffull / f);
        fc[s] = (int32_t)((f << 12) | m->cum[s]);
    }
}

static inline int read_word(const uint8_t *src, size_t len, size_t *sp, uint16_t *w) {
    if (*sp + 2 > len) return ORC_E_TRUNCATED_RENORM;
    *w = (uint16_t)(src[*sp] | (src[*sp + 1] << 8));
    *sp += 2;
    return ORC_OK;
}

/* The scalar encode step (scalar.rs:120-127), specialised to the magic form
 * for the tail; byte-identical to the EncSym form (tested exhaustively). */
static inline void tail_encode(uint32_t *x, uint32_t f, uint32_t c, uint16_t *words, size_t *nw) {
    uint32_t v = *x;
    if ((uint64_t)v >= ((uint64_t)f << 20)) {
        words[(*nw)++] = (uint16_t)(v & 0xffff);
        v >>= 16;
    }
    *x = orc_magic_apply(f, c, v);
}

/* Header parse shared by both SIMD decoders (avx2.rs:58-82). Returns status;
 * *done = 1 for the n == 0 early return. */
static int parse_o0(const uint8_t *src, size_t len, size_t cap, model0 *m, uint32_t *st,
                    size_t *sp, uint64_t *n, int *done) {
    *done = 0;
    if (len < 9) return ORC_E_TRUNCATED;
    uint64_t x = 0;
    for (int i = 8; i >= 1; i--) x = (x << 8) | src[i];
    *n = x;
    if (x == 0) {
        *done = 1;
        return ORC_OK;
    }
    size_t p = 9;
    for (int s = 0; s < 256; s++, p += 2) {
        if (p + 2 > len) return ORC_E_TRUNCATED;
        m->freq[s] = (uint16_t)(src[p] | (src[p + 1] << 8));
    }
    int e = orc_validate_freqs(m->freq);
    if (e) return e;
    model_from_freqs(m);
    for (int i = 0; i < ORC_N_STATES; i++, p += 4) {
        if (p + 4 > len) return ORC_E_TRUNCATED;
        st[i] = (uint32_t)src[p] | ((uint32_t)src[p + 1] << 8) | ((uint32_t)src[p + 2] << 16) |
                ((uint32_t)src[p + 3] << 24);
    }
    if (x > cap) return ORC_E_ALLOC;
    *sp = p;
    return ORC_OK;
}

/* avx2.rs:90-103 / avx512.rs:61-73 */
static int decode_tail(const model0 *m, uint32_t *st, uint8_t *out, size_t from, size_t n,
                       const uint8_t *src, size_t len, size_t *sp) {
    for (size_t i = from; i < n; i++) {
        uint32_t *x = &st[i % ORC_N_STATES];
        uint32_t slot = *x & (ORC_TOTFREQ - 1);
        uint8_t s = m->slot2sym[slot];
        out[i] = s;
        uint32_t v = m->freq[s] * (*x >> ORC_SCALE_BITS) + slot - m->cum[s];
        while (v < ORC_RANS_L) {
            uint16_t w;
            if (read_word(src, len, sp, &w)) return ORC_E_TRUNCATED_RENORM;
            v = (v << 16) | w;
        }
        *x = v;
    }
    return ORC_OK;
}

/* ------------------------------- AVX2 ------------------------------------ */

__attribute__((target("avx2"))) static int load_words8(const uint8_t *src, size_t len,
                                                       size_t *sp, int k, __m256i *out) {
    size_t end = *sp + 2 * (size_t)k;
    if (end > len) return ORC_E_TRUNCATED_RENORM;
    if (*sp + 16 <= len) {
        *out = _mm256_cvtepu16_epi32(_mm_loadu_si128((const __m128i *)(src + *sp)));
    } else {
        uint16_t buf[8] = {0};
        for (int j = 0; j < k; j++) buf[j] = (uint16_t)(src[*sp + 2 * j] | (src[*sp + 2 * j + 1] << 8));
        *out = _mm256_cvtepu16_epi32(_mm_loadu_si128((const __m128i *)buf));
    }
    *sp = end;
    return ORC_OK;
}

/* avx2.rs:130-198 */
__attribute__((target("avx2"))) static int decode_rounds_avx2(const int32_t *packed, uint32_t *st,
                                                              uint8_t *out, const uint8_t *src,
                                                              size_t len, size_t *sp,
                                                              size_t full_rounds) {
    static int32_t perm[256][8];
    static int perm_init = 0;
    if (!perm_init) { /* avx2.rs:111-127 */
        for (int mask = 0; mask < 256; mask++) {
            int rank = 0;
            for (int i = 0; i < 8; i++) {
                perm[mask][i] = 0;
                if ((mask >> i) & 1) perm[mask][i] = rank++;
            }
        }
        perm_init = 1;
    }
    const __m256i mask12 = _mm256_set1_epi32(ORC_TOTFREQ - 1);
    const __m256i mask_off = _mm256_set1_epi32(0xfff);
    const __m256i mask_sym = _mm256_set1_epi32(0xff);
    const __m256i one = _mm256_set1_epi32(1);
    for (size_t round = 0; round < full_rounds; round++) {
        size_t base = round * ORC_N_STATES;
        for (int g = 0; g < ORC_N_STATES / 8; g++) {
            int off = g * 8;
            __m256i v = _mm256_loadu_si256((const __m256i *)(st + off));
            __m256i slot = _mm256_and_si256(v, mask12);
            __m256i p = _mm256_i32gather_epi32((const int *)packed, slot, 4);
            __m256i f = _mm256_add_epi32(_mm256_srli_epi32(p, 20), one);
            __m256i offset = _mm256_and_si256(_mm256_srli_epi32(p, 8), mask_off);
            __m256i sym = _mm256_and_si256(p, mask_sym);
            __m256i vsh = _mm256_srli_epi32(v, ORC_SCALE_BITS);
            __m256i v2 = _mm256_add_epi32(_mm256_mullo_epi32(f, vsh), offset);
            __m256i need = _mm256_cmpeq_epi32(_mm256_srli_epi32(v2, 16), _mm256_setzero_si256());
            int m = _mm256_movemask_ps(_mm256_castsi256_ps(need));
            int k = __builtin_popcount((unsigned)m);
            __m256i renormed = v2;
            if (k) {
                __m256i words;
                if (load_words8(src, len, sp, k, &words)) return ORC_E_TRUNCATED_RENORM;
                __m256i idx = _mm256_loadu_si256((const __m256i *)perm[m]);
                __m256i placed = _mm256_permutevar8x32_epi32(words, idx);
                __m256i shifted = _mm256_or_si256(_mm256_slli_epi32(v2, 16), placed);
                renormed = _mm256_blendv_epi8(v2, shifted, need);
            }
            _mm256_storeu_si256((__m256i *)(st + off), renormed);
            int32_t symtmp[8];
            _mm256_storeu_si256((__m256i *)symtmp, sym);
            for (int l = 0; l < 8; l++) out[base + off + l] = (uint8_t)symtmp[l];
        }
    }
    return ORC_OK;
}

__attribute__((target("avx2"))) static inline __m256i mulhi_epu32_avx2(__m256i a, __m256i b) {
    __m256i evn = _mm256_mul_epu32(a, b);
    __m256i odd = _mm256_mul_epu32(_mm256_srli_epi64(a, 32), _mm256_srli_epi64(b, 32));
    __m256i evn_hi = _mm256_srli_epi64(evn, 32);
    __m256i odd_hi = _mm256_slli_epi64(_mm256_srli_epi64(odd, 32), 32);
    return _mm256_blend_epi32(evn_hi, odd_hi, 0xAA);
}

/* avx2.rs:324-399 */
__attribute__((target("avx2"))) static void encode_rounds_avx2(const int32_t *magic,
                                                               const int32_t *fcs, uint32_t *st,
                                                               const uint8_t *src, uint16_t *words,
                                                               size_t *nw, size_t full_rounds) {
    const __m256i mask12 = _mm256_set1_epi32(0xfff);
    const __m256i mask16 = _mm256_set1_epi32(0xffff);
    const __m256i one = _mm256_set1_epi32(1);
    const __m256i sign = _mm256_set1_epi32((int)0x80000000u);
    for (size_t round = full_rounds; round-- > 0;) {
        size_t base = round * ORC_N_STATES;
        for (int g = ORC_N_STATES / 8 - 1; g >= 0; g--) {
            int off = g * 8;
            __m256i syms = _mm256_cvtepu8_epi32(_mm_loadl_epi64((const __m128i *)(src + base + off)));
            __m256i m = _mm256_i32gather_epi32((const int *)magic, syms, 4);
            __m256i fc = _mm256_i32gather_epi32((const int *)fcs, syms, 4);
            __m256i freq = _mm256_srli_epi32(fc, 12);
            __m256i cum = _mm256_and_si256(fc, mask12);
            __m256i v0 = _mm256_loadu_si256((const __m256i *)(st + off));
            __m256i xmax_m1 = _mm256_sub_epi32(_mm256_slli_epi32(freq, 20), one);
            __m256i need = _mm256_cmpgt_epi32(_mm256_xor_si256(v0, sign), _mm256_xor_si256(xmax_m1, sign));
            __m256i wv = _mm256_and_si256(v0, mask16);
            __m256i v = _mm256_blendv_epi8(v0, _mm256_srli_epi32(v0, 16), need);
            unsigned mask = (unsigned)_mm256_movemask_ps(_mm256_castsi256_ps(need));
            if (mask) {
                int32_t wt[8];
                _mm256_storeu_si256((__m256i *)wt, wv);
                while (mask) {
                    int l = 31 - __builtin_clz(mask);
                    words[(*nw)++] = (uint16_t)wt[l];
                    mask &= ~(1u << l);
                }
            }
            __m256i q0 = mulhi_epu32_avx2(v, m);
            __m256i r0 = _mm256_sub_epi32(v, _mm256_mullo_epi32(q0, freq));
            __m256i ge = _mm256_cmpgt_epi32(r0, _mm256_sub_epi32(freq, one));
            __m256i q = _mm256_sub_epi32(q0, ge);
            __m256i r = _mm256_sub_epi32(r0, _mm256_and_si256(ge, freq));
            __m256i x = _mm256_add_epi32(_mm256_add_epi32(_mm256_slli_epi32(q, ORC_SCALE_BITS), r), cum);
            _mm256_storeu_si256((__m256i *)(st + off), x);
        }
    }
}

/* ------------------------------ AVX-512 ---------------------------------- */

__attribute__((target("avx512f"))) static int load_words16(const uint8_t *src, size_t len,
                                                           size_t *sp, int k, __m512i *out) {
    size_t end = *sp + 2 * (size_t)k;
    if (end > len) return ORC_E_TRUNCATED_RENORM;
    if (*sp + 32 <= len) {
        *out = _mm512_cvtepu16_epi32(_mm256_loadu_si256((const __m256i *)(src + *sp)));
    } else {
        uint16_t buf[16] = {0};
        for (int j = 0; j < k; j++) buf[j] = (uint16_t)(src[*sp + 2 * j] | (src[*sp + 2 * j + 1] << 8));
        *out = _mm512_cvtepu16_epi32(_mm256_loadu_si256((const __m256i *)buf));
    }
    *sp = end;
    return ORC_OK;
}

/* avx512.rs:78-134 */
__attribute__((target("avx512f"))) static int decode_rounds_avx512(const int32_t *packed,
                                                                   uint32_t *st, uint8_t *out,
                                                                   const uint8_t *src, size_t len,
                                                                   size_t *sp, size_t full_rounds) {
    const __m512i mask12 = _mm512_set1_epi32(ORC_TOTFREQ - 1);
    const __m512i mask_off = _mm512_set1_epi32(0xfff);
    const __m512i mask_sym = _mm512_set1_epi32(0xff);
    const __m512i one = _mm512_set1_epi32(1);
    const __m512i rans_l = _mm512_set1_epi32((int)ORC_RANS_L);
    for (size_t round = 0; round < full_rounds; round++) {
        size_t base = round * ORC_N_STATES;
        for (int g = 0; g < 2; g++) {
            int off = g * 16;
            __m512i v = _mm512_loadu_si512((const void *)(st + off));
            __m512i slot = _mm512_and_si512(v, mask12);
            __m512i p = _mm512_i32gather_epi32(slot, (const void *)packed, 4);
            __m512i f = _mm512_add_epi32(_mm512_srli_epi32(p, 20), one);
            __m512i offset = _mm512_and_si512(_mm512_srli_epi32(p, 8), mask_off);
            __m512i sym = _mm512_and_si512(p, mask_sym);
            __m512i vsh = _mm512_srli_epi32(v, ORC_SCALE_BITS);
            __m512i v2 = _mm512_add_epi32(_mm512_mullo_epi32(f, vsh), offset);
            __mmask16 need = _mm512_cmplt_epu32_mask(v2, rans_l);
            int k = __builtin_popcount((unsigned)need);
            __m512i renormed = v2;
            if (k) {
                __m512i words;
                if (load_words16(src, len, sp, k, &words)) return ORC_E_TRUNCATED_RENORM;
                __m512i expanded = _mm512_maskz_expand_epi32(need, words);
                __m512i shifted = _mm512_or_si512(_mm512_slli_epi32(v2, 16), expanded);
                renormed = _mm512_mask_blend_epi32(need, v2, shifted);
            }
            _mm512_storeu_si512((void *)(st + off), renormed);
            _mm_storeu_si128((__m128i *)(out + base + off), _mm512_cvtepi32_epi8(sym));
        }
    }
    return ORC_OK;
}

__attribute__((target("avx512f"))) static inline __m512i mulhi_epu32_512(__m512i a, __m512i b) {
    __m512i evn = _mm512_mul_epu32(a, b);
    __m512i odd = _mm512_mul_epu32(_mm512_srli_epi64(a, 32), _mm512_srli_epi64(b, 32));
    __m512i evn_hi = _mm512_srli_epi64(evn, 32);
    __m512i odd_hi = _mm512_slli_epi64(_mm512_srli_epi64(odd, 32), 32);
    return _mm512_mask_blend_epi32(0xAAAA, evn_hi, odd_hi);
}

/* avx512.rs:213-282 */
__attribute__((target("avx512f"))) static void encode_rounds_avx512(const int32_t *magic,
                                                                    const int32_t *fcs,
                                                                    uint32_t *st,
                                                                    const uint8_t *src,
                                                                    uint16_t *words, size_t *nw,
                                                                    size_t full_rounds) {
    const __m512i mask12 = _mm512_set1_epi32(0xfff);
    const __m512i mask16 = _mm512_set1_epi32(0xffff);
    const __m512i one = _mm512_set1_epi32(1);
    for (size_t round = full_rounds; round-- > 0;) {
        size_t base = round * ORC_N_STATES;
        for (int g = 1; g >= 0; g--) {
            int off = g * 16;
            __m512i syms = _mm512_cvtepu8_epi32(_mm_loadu_si128((const __m128i *)(src + base + off)));
            __m512i m = _mm512_i32gather_epi32(syms, (const void *)magic, 4);
            __m512i fc = _mm512_i32gather_epi32(syms, (const void *)fcs, 4);
            __m512i freq = _mm512_srli_epi32(fc, 12);
            __m512i cum = _mm512_and_si512(fc, mask12);
            __m512i v0 = _mm512_loadu_si512((const void *)(st + off));
            __m512i xmax_m1 = _mm512_sub_epi32(_mm512_slli_epi32(freq, 20), one);
            __mmask16 need = _mm512_cmpgt_epu32_mask(v0, xmax_m1);
            __m512i wv = _mm512_and_si512(v0, mask16);
            __m512i v = _mm512_mask_srli_epi32(v0, need, v0, 16);
            unsigned mask = (unsigned)need;
            if (mask) {
                int32_t wt[16];
                _mm512_storeu_si512((void *)wt, wv);
                while (mask) {
                    int l = 31 - __builtin_clz(mask);
                    words[(*nw)++] = (uint16_t)wt[l];
                    mask &= ~(1u << l);
                }
            }
            __m512i q0 = mulhi_epu32_512(v, m);
            __m512i r0 = _mm512_sub_epi32(v, _mm512_mullo_epi32(q0, freq));
            __mmask16 ge = _mm512_cmpge_epu32_mask(r0, freq);
            __m512i q = _mm512_mask_add_epi32(q0, ge, q0, one);
            __m512i r = _mm512_mask_sub_epi32(r0, ge, r0, freq);
            __m512i x = _mm512_add_epi32(_mm512_add_epi32(_mm512_slli_epi32(q, ORC_SCALE_BITS), r), cum);
            _mm512_storeu_si512((void *)(st + off), x);
        }
    }
}

/* ------------------------- public SIMD entry points ---------------------- */

/* avx2.rs:269-307 / avx512.rs:164-198 */
int orc_encode_o0_simd(int level, const uint8_t *src, size_t n, uint8_t *dst, size_t dst_cap,
                       size_t *out_len) {
    if (level < 1 || level > orc_simd_level()) return ORC_E_INVALID_ARG;
    if (dst_cap < orc_encode_bound(n, 0)) return ORC_E_DST_TOO_SMALL;
    model0 m;
    uint32_t counts[256] = {0};
    for (size_t i = 0; i < n; i++) counts[src[i]]++;
    orc_normalize(counts, m.freq);
    model_from_freqs(&m);
    int32_t magic[256], fc[256];
    enc_tables(&m, magic, fc);
    uint32_t st[ORC_N_STATES];
    for (int i = 0; i < ORC_N_STATES; i++) st[i] = ORC_RANS_L;
    uint16_t *words = n ? (uint16_t *)malloc(n * sizeof(uint16_t)) : NULL;
    size_t nw = 0;
    size_t full = n / ORC_N_STATES;
    for (size_t i = n; i-- > full * ORC_N_STATES;) {
        uint8_t s = src[i];
        tail_encode(&st[i % ORC_N_STATES], m.freq[s], m.cum[s], words, &nw);
    }
    if (level == 2)
        encode_rounds_avx512(magic, fc, st, src, words, &nw, full);
    else
        encode_rounds_avx2(magic, fc, st, src, words, &nw, full);
    size_t o = 0;
    dst[o++] = 0;
    for (int i = 0; i < 8; i++) dst[o++] = (uint8_t)((uint64_t)n >> (8 * i));
    if (n) {
        for (int s = 0; s < 256; s++, o += 2) {
            dst[o] = (uint8_t)m.freq[s];
            dst[o + 1] = (uint8_t)(m.freq[s] >> 8);
        }
        o += orc__finish(dst + o, st, words, nw);
    }
    free(words);
    *out_len = o;
    return ORC_OK;
}

/* avx2.rs:58-105 / avx512.rs:29-75 */
int orc_decode_o0_simd(int level, const uint8_t *src, size_t len, uint8_t *dst, size_t dst_cap,
                       size_t *out_len) {
    if (level < 1 || level > orc_simd_level()) return ORC_E_INVALID_ARG;
    model0 m;
    uint32_t st[ORC_N_STATES];
    size_t sp = 0;
    uint64_t n = 0;
    int done;
    *out_len = 0;
    int e = parse_o0(src, len, dst_cap, &m, st, &sp, &n, &done);
    if (e || done) return e;
    int32_t *packed = (int32_t *)malloc(ORC_TOTFREQ * sizeof(int32_t));
    slot_table(&m, packed);
    size_t full = (size_t)n / ORC_N_STATES;
    e = level == 2 ? decode_rounds_avx512(packed, st, dst, src, len, &sp, full)
                   : decode_rounds_avx2(packed, st, dst, src, len, &sp, full);
    free(packed);
    if (e) return e;
    e = decode_tail(&m, st, dst, full * ORC_N_STATES, (size_t)n, src, len, &sp);
    if (!e) *out_len = (size_t)n;
    return e;
}

/* --------------------- block-parallel batch driver ----------------------- */

typedef struct {
    const uint8_t *src;
    const uint64_t *src_off, *src_len;
    size_t nblocks;
    int order, decode;
    uint8_t *dst;
    const uint64_t *dst_off, *dst_cap;
    uint64_t *out_len;
    int32_t *status;
    atomic_size_t next;
} batch_job;

static void *batch_worker(void *arg) {
    batch_job *J = (batch_job *)arg;
    for (;;) {
        size_t i = atomic_fetch_add(&J->next, 1);
        if (i >= J->nblocks) break;
        const uint8_t *s = J->src + J->src_off[i];
        uint8_t *d = J->dst + J->dst_off[i];
        size_t ol = 0;
        int st;
        if (J->decode) {
            st = orc_decode_dispatch(s, J->src_len[i], d, J->dst_cap[i], &ol);
        } else if (J->order == 2) {
            /* both orders, keep the smaller, ties to order 0 */
            size_t l1 = 0;
            uint8_t *tmp = (uint8_t *)malloc(orc_encode_bound(J->src_len[i], 1));
            st = orc_encode_dispatch(s, J->src_len[i], 0, d, J->dst_cap[i], &ol);
            if (!st && tmp && !orc_encode(s, J->src_len[i], 1, tmp, orc_encode_bound(J->src_len[i], 1), &l1) &&
                l1 < ol) {
                memcpy(d, tmp, l1);
                ol = l1;
            }
            free(tmp);
        } else {
            st = orc_encode_dispatch(s, J->src_len[i], J->order, d, J->dst_cap[i], &ol);
        }
        J->out_len[i] = ol;
        J->status[i] = st;
    }
    return NULL;
}

static int run_batch(batch_job *J, int nthreads) {
    if (nthreads <= 0) nthreads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nthreads < 1) nthreads = 1;
    atomic_init(&J->next, 0);
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nthreads);
    int started = 0;
    for (int t = 1; t < nthreads; t++)
        if (pthread_create(&th[started], NULL, batch_worker, J) == 0) started++;
    batch_worker(J);
    for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
    free(th);
    for (size_t i = 0; i < J->nblocks; i++)
        if (J->status[i]) return J->status[i];
    return ORC_OK;
}

int orc_encode_batch(const uint8_t *src, const uint64_t *src_off, const uint64_t *src_len,
                     size_t nblocks, int order, uint8_t *dst, const uint64_t *dst_off,
                     const uint64_t *dst_cap, uint64_t *out_len, int32_t *status, int nthreads) {
    batch_job J = {src, src_off, src_len, nblocks, order, 0, dst, dst_off, dst_cap, out_len, status};
    return run_batch(&J, nthreads);
}

int orc_decode_batch(const uint8_t *src, const uint64_t *src_off, const uint64_t *src_len,
                     size_t nblocks, uint8_t *dst, const uint64_t *dst_off,
                     const uint64_t *dst_cap, uint64_t *out_len, int32_t *status, int nthreads) {
    batch_job J = {src, src_off, src_len, nblocks, 0, 1, dst, dst_off, dst_cap, out_len, status};
    return run_batch(&J, nthreads);
}
