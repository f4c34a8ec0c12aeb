// The reorder permutation's byte planes (crates/fqxv/src/container/
// reorder.rs:597-609 encode_perm, :1089-1105 decode_permutation) on the GPU:
// the n u32 entries are split into four planes (plane k = byte k of every
// entry) by a kernel, the 4 n bytes coded as one stream by the batch coder,
// and the reverse on decode.
#include <algorithm>

#include "../../include/fqxv_streams_gpu.h"
#include "rans_ctx.cuh"

using namespace fqxv;

namespace {

// Four entries a thread: one 16-byte load, four 4-byte plane stores.
__global__ void perm_planes_kernel(const uint32_t *order, uint64_t n, uint8_t *planes) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = 4 * ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x); i < n; i += 4 * stride) {
        uint32_t v[4] = {0, 0, 0, 0};
        const int m = n - i < 4 ? (int)(n - i) : 4;
        for (int j = 0; j < m; j++) v[j] = order[i + j];
        for (int k = 0; k < 4; k++)
            for (int j = 0; j < m; j++) planes[k * n + i + j] = (uint8_t)(v[j] >> (8 * k));
    }
}

__global__ void perm_join_kernel(const uint8_t *planes, uint64_t n, uint32_t *order) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        order[i] = (uint32_t)planes[i] | (uint32_t)planes[n + i] << 8 | (uint32_t)planes[2 * n + i] << 16 |
                   (uint32_t)planes[3 * n + i] << 24;
}

int grid_for(fqxv_rans_ctx *ctx, uint64_t n) {
    return (int)std::max<uint64_t>(1, std::min<uint64_t>((n + 1023) / 1024, (uint64_t)ctx->sms * 8));
}

}  // namespace

extern "C" {

int fqxv_perm_encode_host(fqxv_rans_ctx *ctx, const uint32_t *order, uint64_t n, uint8_t *h_dst, uint64_t cap,
                          uint64_t *out_len) {
    if (!ctx || !h_dst || !out_len || (n && !order) || n > (1ull << 60)) return FQXV_RANS_E_INVALID_ARG;
    std::lock_guard<std::mutex> g(ctx->mu);
    DeviceGuard dg(ctx->device);
    cudaStream_t s = ctx->stream;
    const uint64_t nb = 4 * n, ocap = 9 + 512 + 128 + 2 * nb;  // the smaller order fits the order-0 bound
    CK(ctx->io_in.ensure(std::max<uint64_t>(2 * nb, 16), s));
    CK(ctx->io_out.ensure(std::max<uint64_t>(ocap, 16), s));
    uint32_t *d_order = ctx->io_in.as<uint32_t>();
    uint8_t *d_planes = ctx->io_in.as<uint8_t>() + nb;
    uint8_t *d_out = ctx->io_out.as<uint8_t>();
    if (n) {
        CK(cudaMemcpyAsync(d_order, order, nb, cudaMemcpyHostToDevice, s));
        perm_planes_kernel<<<grid_for(ctx, n / 4 + 1), 256, 0, s>>>(d_order, n, d_planes);
        CK(cudaGetLastError());
    }
    // reorder.rs:604-606: both orders, the smaller kept, ties to order-0
    fqxv_rans_span sp{0, nb}, os{0, 0};
    const int st = encode_batch_locked(ctx, d_planes, &sp, 1, FQXV_RANS_BEST_TIE0, d_out, ocap, &os, nullptr);
    if (st) return st;
    *out_len = os.length;
    if (os.length > cap) return FQXV_RANS_E_DST_TOO_SMALL;
    CK(cudaMemcpyAsync(h_dst, d_out + os.offset, os.length, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return FQXV_RANS_OK;
}

int fqxv_perm_decode_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, uint64_t len, uint64_t n, uint32_t *order) {
    if (!ctx || (len && !h_src) || (n && !order) || n > (1ull << 60)) return FQXV_RANS_E_INVALID_ARG;
    std::lock_guard<std::mutex> g(ctx->mu);
    DeviceGuard dg(ctx->device);
    cudaStream_t s = ctx->stream;
    const uint64_t nb = 4 * n;
    CK(ctx->io_in.ensure(std::max<uint64_t>(len, 16), s));
    CK(ctx->io_out.ensure(2 * nb + 16, s));  // planes, then the entries 16-byte aligned
    uint8_t *d_src = ctx->io_in.as<uint8_t>();
    uint8_t *d_planes = ctx->io_out.as<uint8_t>();
    if (len) CK(cudaMemcpyAsync(d_src, h_src, len, cudaMemcpyHostToDevice, s));
    // reorder.rs:1097-1101: decode_bounded(perm_c, 4 n), then exactly 4 n bytes
    fqxv_rans_span sp{0, len}, os{0, nb};
    uint64_t got = 0;
    int32_t ds = 0;
    const int st = decode_batch_locked(ctx, d_src, &sp, 1, nb, d_planes, &os, &got, &ds);
    if (st != FQXV_RANS_OK && !(st >= FQXV_RANS_E_TRUNCATED && st <= FQXV_RANS_E_TRUNCATED_RENORM)) return st;
    if (ds != FQXV_RANS_OK) return FQXV_PERM_E_BAD;
    if (got != nb) return FQXV_PERM_E_LENGTH;
    if (!n) return FQXV_RANS_OK;
    uint32_t *d_order = reinterpret_cast<uint32_t *>(d_planes + nb + ((16 - (nb & 15)) & 15));
    perm_join_kernel<<<grid_for(ctx, n), 256, 0, s>>>(d_planes, n, d_order);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(order, d_order, nb, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return FQXV_RANS_OK;
}

}  // extern "C"
