/*
 * TEST INFRASTRUCTURE ONLY: the two batch-coder entry points the tokenizer
 * host code (fqxv_b200/csrc/tok_capi.cu) calls, restated over the CPU oracle
 * and run on host threads (one stream at a time per thread, as the
 * reference's callers code blocks on rayon workers). Linked with tok_capi.cu
 * into oracle/_build/libcallers_cpu.so, which the tests use to check the
 * tokenizer's host logic against the oracle tokenizer without a GPU and
 * bench.py times as the CPU baseline of the names workload. The product
 * library links the GPU coder instead.
 */
#include <pthread.h>
#include <stdatomic.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "../include/fqxv_rans_gpu.h"
#include "rans_oracle.h"

typedef struct {
    const uint8_t *src;
    const fqxv_rans_span *blocks;
    size_t n;
    int order;
    uint8_t **enc;
    size_t *enc_len;
    int32_t *st;
    atomic_size_t next;
    /* decode */
    uint64_t max_len;
    uint8_t *dst;
    const fqxv_rans_span *out;
    uint64_t *out_len;
} job_t;

static void *enc_worker(void *arg) {
    job_t *J = (job_t *)arg;
    for (;;) {
        const size_t i = atomic_fetch_add(&J->next, 1);
        if (i >= J->n) break;
        const uint8_t *s = J->src + J->blocks[i].offset;
        const size_t n = J->blocks[i].length;
        const size_t cap0 = orc_encode_bound(n, 0), cap1 = orc_encode_bound(n, 1);
        uint8_t *e0 = (uint8_t *)malloc(cap0), *e1 = J->order != FQXV_RANS_ORDER0 ? (uint8_t *)malloc(cap1) : NULL;
        size_t l0 = 0, l1 = 0;
        int st = orc_encode(s, n, 0, e0, cap0, &l0);
        if (!st && e1) st = orc_encode(s, n, 1, e1, cap1, &l1);
        J->st[i] = st;
        if (!e1 || (J->order == FQXV_RANS_BEST_TIE0 && l1 >= l0) || (J->order == FQXV_RANS_BEST_TIE1 && l1 > l0)) {
            J->enc[i] = e0;
            J->enc_len[i] = l0;
            free(e1);
        } else {
            J->enc[i] = e1;
            J->enc_len[i] = l1;
            free(e0);
        }
    }
    return NULL;
}

static void *dec_worker(void *arg) {
    job_t *J = (job_t *)arg;
    for (;;) {
        const size_t i = atomic_fetch_add(&J->next, 1);
        if (i >= J->n) break;
        size_t ol = 0;
        const int st = orc_decode_bounded(J->src + J->blocks[i].offset, J->blocks[i].length, (size_t)J->max_len,
                                          J->dst + J->out[i].offset, J->out[i].length, &ol);
        J->st[i] = st;
        J->out_len[i] = st ? 0 : ol;
    }
    return NULL;
}

static void run(job_t *J, void *(*fn)(void *)) {
    long nt = sysconf(_SC_NPROCESSORS_ONLN);
    if (nt < 1) nt = 1;
    if ((size_t)nt > J->n) nt = (long)(J->n ? J->n : 1);
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nt);
    long started = 0;
    for (long t = 0; t < nt; t++)
        if (pthread_create(&th[started], NULL, fn, J) == 0) started++;
    if (!started) fn(J);
    for (long t = 0; t < started; t++) pthread_join(th[t], NULL);
    free(th);
}

int fqxv_rans_encode_batch_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, const fqxv_rans_span *blocks,
                                size_t nblocks, int order, uint8_t *h_dst, uint64_t dst_cap,
                                fqxv_rans_span *out_spans, int32_t *out_orders) {
    (void)ctx;
    job_t J;
    memset(&J, 0, sizeof J);
    J.src = h_src;
    J.blocks = blocks;
    J.n = nblocks;
    J.order = order;
    J.enc = (uint8_t **)calloc(nblocks ? nblocks : 1, sizeof(uint8_t *));
    J.enc_len = (size_t *)calloc(nblocks ? nblocks : 1, sizeof(size_t));
    J.st = (int32_t *)calloc(nblocks ? nblocks : 1, sizeof(int32_t));
    run(&J, enc_worker);
    int rc = FQXV_RANS_OK;
    uint64_t pos = 0;
    for (size_t i = 0; i < nblocks; i++) {
        if (!rc && J.st[i]) rc = J.st[i];
        if (!rc && pos + J.enc_len[i] > dst_cap) rc = FQXV_RANS_E_DST_TOO_SMALL;
        if (!rc) {
            memcpy(h_dst + pos, J.enc[i], J.enc_len[i]);
            out_spans[i].offset = pos;
            out_spans[i].length = J.enc_len[i];
            if (out_orders) out_orders[i] = J.enc[i][0];
            pos += J.enc_len[i];
        }
        free(J.enc[i]);
    }
    free(J.enc);
    free(J.enc_len);
    free(J.st);
    return rc;
}

int fqxv_rans_decode_batch_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, const fqxv_rans_span *blocks,
                                size_t nblocks, uint64_t max_len, uint8_t *h_dst,
                                const fqxv_rans_span *out_spans, uint64_t *out_lens, int32_t *status) {
    (void)ctx;
    job_t J;
    memset(&J, 0, sizeof J);
    J.src = h_src;
    J.blocks = blocks;
    J.n = nblocks;
    J.max_len = max_len;
    J.dst = h_dst;
    J.out = out_spans;
    J.out_len = out_lens;
    J.st = status;
    run(&J, dec_worker);
    for (size_t i = 0; i < nblocks; i++)
        if (status[i]) return status[i];
    return FQXV_RANS_OK;
}
