// Warp-level helpers shared by the encode and decode kernels.
#pragma once

#include <stdint.h>

namespace fqxv {

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Predicated stores: no branch, so unrolled rounds stay one basic block.
__device__ __forceinline__ void st_u16_if(bool p, uint16_t *addr, uint32_t v) {
    asm volatile(
        "{\n .reg .pred q;\n setp.ne.b32 q, %0, 0;\n @q st.global.u16 [%1], %2;\n}" ::"r"((int)p), "l"(addr),
        "h"((unsigned short)v)
        : "memory");
}

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Inclusive warp scan of u32.
__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

__device__ __forceinline__ uint64_t warp_incl_scan_u64(uint64_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

__device__ __forceinline__ uint32_t ld_u32_le(const uint8_t *p) {
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

__device__ __forceinline__ uint64_t ld_u64_le(const uint8_t *p) {
    uint64_t v = 0;
#pragma unroll
    for (int i = 7; i >= 0; i--) v = (v << 8) | p[i];
    return v;
}

// Normalise m (<= 256) counts, held in ascending symbol order, into
// frequencies summing to 4096 with the reference's rounding and tie rules
// (crates/fqxv-rans/src/model.rs:213-264):
//   f = max(1, c * 4096 / total) for every occurring symbol;
//   max_s = first symbol with the strictly largest f;
//   a positive residual goes to max_s; a negative one drains max_s down to 1,
//   then re-picks the first symbol with the strictly largest f > 1, repeating.
// One warp; lane l owns entries [8l, 8l + 8). Also returns the exclusive
// cumulative frequency of each entry. `present` is false for an all-zero row.
__device__ __forceinline__ void warp_normalize(const uint32_t *counts, int m, uint32_t f[8],
                                               uint32_t cum[8], bool &present) {
    const int lane = threadIdx.x & 31;
    uint32_t c[8];
    uint64_t tot = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int idx = lane * 8 + k;
        c[k] = idx < m ? counts[idx] : 0u;
        tot += c[k];
    }
    tot = warp_sum_u64(tot);
    present = tot != 0;
    if (!present) {
#pragma unroll
        for (int k = 0; k < 8; k++) f[k] = cum[k] = 0;
        return;
    }
    uint32_t sum = 0, key = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const uint32_t idx = lane * 8 + k;
        uint32_t v = 0;
        if (c[k]) {
            v = (uint32_t)(((uint64_t)c[k] * 4096u) / tot);
            if (v == 0) v = 1;
        }
        f[k] = v;
        sum += v;
        const uint32_t kk = v ? (v << 9) | (511u - idx) : 0u;
        key = kk > key ? kk : key;
    }
    sum = __reduce_add_sync(0xffffffffu, sum);
    key = __reduce_max_sync(0xffffffffu, key);
    int max_s = 511 - (int)(key & 511u);
    int diff = 4096 - (int)sum;
    if (diff > 0) {
#pragma unroll
        for (int k = 0; k < 8; k++)
            if (lane * 8 + k == max_s) f[k] += (uint32_t)diff;
    } else {
        // At most one pass per occurring symbol; the guard only bounds the loop.
        for (int iter = 0; diff < 0 && iter < 512; iter++) {
            uint32_t take = 0;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                if (lane * 8 + k == max_s) {
                    take = f[k] - 1u;
                    if (take > (uint32_t)(-diff)) take = (uint32_t)(-diff);
                    f[k] -= take;
                }
            }
            take = __reduce_add_sync(0xffffffffu, take);
            diff += (int)take;
            if (diff != 0) {
                key = 0;
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const uint32_t idx = lane * 8 + k;
                    const uint32_t kk = f[k] > 1u ? (f[k] << 9) | (511u - idx) : 0u;
                    key = kk > key ? kk : key;
                }
                key = __reduce_max_sync(0xffffffffu, key);
                if (key == 0) break;
                max_s = 511 - (int)(key & 511u);
            }
        }
    }
    uint32_t local = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        cum[k] = local;
        local += f[k];
    }
    const uint32_t excl = warp_incl_scan(local) - local;
#pragma unroll
    for (int k = 0; k < 8; k++) cum[k] += excl;
}

}  // namespace fqxv
