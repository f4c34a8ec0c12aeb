/*
 * TEST INFRASTRUCTURE ONLY: the two batch-coder entry points the tokenizer
 * (fqxv_b200/csrc/tok_capi.cu) calls, restated over the CPU oracle, so that the
 * tokenizer's host logic -- role streams, op runs, byte planes, payload
 * framing, error order -- can be checked against the oracle tokenizer on a
 * machine without a GPU. Linked only into tests/_build/libtokcheck.so by
 * tests/test_tok_cpu.py; the product library links the real GPU coder.
 */
#include <stdint.h>
#include <string.h>

#include "../../include/fqxv_rans_gpu.h"
#include "../../oracle/rans_oracle.h"

int fqxv_rans_encode_batch_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, const fqxv_rans_span *blocks,
                                size_t nblocks, int order, uint8_t *h_dst, uint64_t dst_cap,
                                fqxv_rans_span *out_spans, int32_t *out_orders) {
    (void)ctx;
    static uint8_t e0[1 << 22], e1[(1 << 22) + 140000];
    uint64_t pos = 0;
    for (size_t i = 0; i < nblocks; i++) {
        size_t l0 = 0, l1 = 0;
        const uint8_t *s = h_src + blocks[i].offset;
        if (blocks[i].length > (1 << 21)) return FQXV_RANS_E_TOO_LARGE;
        int st = orc_encode(s, blocks[i].length, 0, e0, sizeof e0, &l0);
        if (st) return st;
        const uint8_t *pick = e0;
        size_t pl = l0;
        int po = 0;
        if (order != FQXV_RANS_ORDER0) {
            st = orc_encode(s, blocks[i].length, 1, e1, sizeof e1, &l1);
            if (st) return st;
            if (order == FQXV_RANS_ORDER1 || l1 < l0 || (order == FQXV_RANS_BEST_TIE1 && l1 == l0)) {
                pick = e1;
                pl = l1;
                po = 1;
            }
        }
        if (pos + pl > dst_cap) return FQXV_RANS_E_DST_TOO_SMALL;
        memcpy(h_dst + pos, pick, pl);
        out_spans[i].offset = pos;
        out_spans[i].length = pl;
        if (out_orders) out_orders[i] = po;
        pos += pl;
    }
    return FQXV_RANS_OK;
}

int fqxv_rans_decode_batch_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, const fqxv_rans_span *blocks,
                                size_t nblocks, uint64_t max_len, uint8_t *h_dst,
                                const fqxv_rans_span *out_spans, uint64_t *out_lens, int32_t *status) {
    (void)ctx;
    int first = FQXV_RANS_OK;
    for (size_t i = 0; i < nblocks; i++) {
        size_t ol = 0;
        const int st = orc_decode_bounded(h_src + blocks[i].offset, blocks[i].length, (size_t)max_len,
                                          h_dst + out_spans[i].offset, out_spans[i].length, &ol);
        status[i] = st;
        out_lens[i] = st ? 0 : ol;
        if (st && first == FQXV_RANS_OK) first = st;
    }
    return first;
}
