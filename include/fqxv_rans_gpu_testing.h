/*
 * fqxv_rans_gpu_testing.h -- test-only controls of libfqxv_rans_gpu.so.
 *
 * Not part of the coder's API (fqxv_rans_gpu.h) and with no counterpart in
 * the reference: these calls exist so that tests can drive failure paths that
 * normal operation never reaches, without faulting or hanging a GPU.
 */
#ifndef FQXV_RANS_GPU_TESTING_H
#define FQXV_RANS_GPU_TESTING_H

#include <stdint.h>

#include "fqxv_rans_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Polls a decode kernel makes of its table copy's barrier before it gives up
 * (default 4194304). A wait that gives up is followed by a drain of the same
 * copy with the default bound; the stream then reports FQXV_RANS_E_TIMEOUT,
 * and a CTA whose drain also failed reports FQXV_RANS_E_TIMEOUT for every
 * stream it takes afterwards without issuing another copy. 0 makes every
 * first wait give up at once, so each stream of the order-0 and shared-memory
 * order-1 decoders reports FQXV_RANS_E_TIMEOUT while its copy still lands.
 * Applies to the context and its sub-contexts. */
int fqxv_rans_ctx_test_set_wait_polls(fqxv_rans_ctx *ctx, uint32_t polls);

#ifdef __cplusplus
}
#endif
#endif
