/* A plain C99 caller of the library: encodes a buffer at both orders through
 * the single-call C ABI, decodes it back, checks the bytes, and checks that a
 * bounded decode of a stream longer than the bound fails with the
 * reference's error -- what a Rust, Go or C binding does through FFI.
 * Exit status 0 on success. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fqxv_rans_gpu.h"

int main(void) {
    const size_t n = 200000;
    uint8_t *src = malloc(n);
    uint32_t z = 7;
    uint8_t q = 30;
    for (size_t i = 0; i < n; i++) {
        z = z * 1664525u + 1013904223u;
        q = (uint8_t)(q + (int)((z >> 28) % 3) - 1);
        if (q < 2) q = 2;
        if (q > 41) q = 41;
        src[i] = (uint8_t)(33 + q);
    }
    for (int order = FQXV_RANS_ORDER0; order <= FQXV_RANS_ORDER1; order++) {
        const size_t cap = fqxv_rans_encode_bound(n, order);
        uint8_t *enc = malloc(cap);
        uint8_t *dec = malloc(n);
        size_t elen = 0, dlen = 0, peek = 0;
        int st = fqxv_rans_encode(src, n, order, enc, cap, &elen);
        if (st) {
            fprintf(stderr, "encode order %d: %s\n", order, fqxv_rans_status_message(st));
            return 1;
        }
        if (enc[0] != order || fqxv_rans_peek_output_len(enc, elen, &peek) || peek != n) {
            fprintf(stderr, "header of order %d stream is wrong\n", order);
            return 1;
        }
        st = fqxv_rans_decode(enc, elen, dec, n, &dlen);
        if (st || dlen != n || memcmp(dec, src, n) != 0) {
            fprintf(stderr, "decode order %d: %s\n", order, st ? fqxv_rans_status_message(st) : "bytes differ");
            return 1;
        }
        st = fqxv_rans_decode_bounded(enc, elen, n - 1, dec, n, &dlen);
        if (st != FQXV_RANS_E_BOUND) {
            fprintf(stderr, "bounded decode: want %d got %d\n", FQXV_RANS_E_BOUND, st);
            return 1;
        }
        printf("order %d: %zu -> %zu bytes, round trip ok\n", order, n, elen);
        free(enc);
        free(dec);
    }
    free(src);
    return 0;
}
