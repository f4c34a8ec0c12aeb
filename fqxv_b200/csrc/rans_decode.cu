// Decode path of the B200 rANS Nx16 coder.
//
//   1. dec_parse_kernel  one CTA per stream: header checks in the reference's
//      order (lib.rs:226-231, scalar.rs:143-217, model.rs:160-205), then the
//      decode tables: order-0 one packed word per slot ((f-1)<<20 | offset<<8
//      | sym, the layout of avx2.rs:29-54); order-1 per present context a
//      slot -> (symbol, dense next context) table and a (freq << 12 | cum)
//      table.
//   2. dec_run_kernel    one warp per stream from a device work queue: lane l
//      owns state l; renorm words are handed out in stream order by a
//      ballot/popc prefix over the lanes that need one. Order-1 resolves the
//      previous-symbol context chain of each round lane by lane.
// Malformed input never faults: every read of the stream is bounds checked
// and errors are reported per stream as the reference's Malformed kinds.
#include "rans_common.cuh"
#include "rans_internal.cuh"

namespace fqxv {

__global__ void __launch_bounds__(kParseThreads)
    dec_parse_kernel(const uint8_t *__restrict__ src, DecStream *__restrict__ streams, int nstreams,
                     uint8_t *__restrict__ tbl) {
    __shared__ uint32_t sfreq[256];
    __shared__ uint32_t scum[257];
    __shared__ uint32_t wsum[kParseThreads / 32];
    __shared__ uint8_t ctxmap[256];
    __shared__ int s_k;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    for (int si = blockIdx.x; si < nstreams; si += gridDim.x) {
        DecStream &S = streams[si];
        const uint8_t *p = src + S.src_off;
        const uint64_t L = S.src_len;
        uint64_t n = 0;
        int order = 0;
        if (L >= 9) {
            order = p[0];
            n = ld_u64_le(p + 1);
        }
        int status = FQXV_RANS_OK;
        if (L >= 9 && n > S.max_len) status = FQXV_RANS_E_BOUND;   // lib.rs:227
        else if (L < 9) status = FQXV_RANS_E_TRUNCATED;             // scalar.rs:145-146
        else if (n != 0 && order > 1) status = FQXV_RANS_E_UNKNOWN_ORDER;
        if (tid == 0) {
            S.order = order;
            S.n = (status == FQXV_RANS_OK) ? n : 0;
            S.nctx = 0;
            S.ctx0 = 0xff;
        }
        if (status != FQXV_RANS_OK || n == 0) {
            if (tid == 0) S.status = status;
            __syncthreads();
            continue;
        }
        uint8_t *T = tbl + S.tbl_off;
        // Validate one 256-entry frequency table at byte offset `at` (the
        // caller checked it is in bounds); fills sfreq/scum. model.rs:160-174.
        auto load_table = [&](uint64_t at) -> int {
            const uint32_t f = tid < 256 ? (uint32_t)p[at + 2 * tid] | ((uint32_t)p[at + 2 * tid + 1] << 8) : 0u;
            if (tid < 256) sfreq[tid] = f;
            const uint32_t incl = warp_incl_scan(f);
            if (lane == 31) wsum[warp] = incl;
            __syncthreads();
            uint32_t base = 0;
            for (int w = 0; w < warp; w++) base += wsum[w];
            if (tid < 256) scum[tid] = base + incl - f;
            uint32_t tot = 0;
            for (int w = 0; w < kParseThreads / 32; w++) tot += wsum[w];
            if (tid == 0) scum[256] = tot;
            __syncthreads();
            // Running sums are monotone, so "some prefix exceeds" == "total exceeds".
            return tot > kTotFreq ? FQXV_RANS_E_FREQ_EXCEEDS
                                  : (tot != kTotFreq ? FQXV_RANS_E_FREQ_SUM : FQXV_RANS_OK);
        };
        uint64_t hdr = 0;
        if (order == 0) {
            if (L < kHdr + kO0Tables) status = FQXV_RANS_E_TRUNCATED;
            else status = load_table(kHdr);
            hdr = kHdr + kO0Tables;
            if (status == FQXV_RANS_OK && L < hdr + kStatesBytes) status = FQXV_RANS_E_TRUNCATED;
            if (status == FQXV_RANS_OK && n > S.dst_cap) status = FQXV_RANS_E_ALLOC;
            if (status == FQXV_RANS_OK) {
                uint32_t *P = reinterpret_cast<uint32_t *>(T);
                for (int slot = tid; slot < (int)kTotFreq; slot += blockDim.x) {
                    // largest s with cum[s] <= slot and f[s] > 0
                    int lo = 0, hi = 255;
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (scum[mid] <= (uint32_t)slot) lo = mid; else hi = mid - 1;
                    }
                    const uint32_t f = sfreq[lo], c = scum[lo];
                    P[slot] = ((f - 1) << 20) | (((uint32_t)slot - c) << 8) | (uint32_t)lo;
                }
            }
        } else {
            if (L < kHdr + kO1Bitmap) {
                status = FQXV_RANS_E_TRUNCATED;
            } else {
                if (warp == 0) {
                    const uint32_t byte = p[kHdr + lane];
                    const uint32_t c = __popc(byte);
                    uint32_t base = warp_incl_scan(c) - c;
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        const int ctx = lane * 8 + k;
                        if ((byte >> k) & 1u) {
                            ctxmap[ctx] = (uint8_t)(base++);
                        } else {
                            ctxmap[ctx] = 0xff;
                        }
                    }
                    if (lane == 31) s_k = (int)base;
                }
                __syncthreads();
                const int K = s_k;
                if (tid < 256) T[kDecCtxMap + tid] = ctxmap[tid];
                for (int t = 0; t < K && status == FQXV_RANS_OK; t++) {
                    const uint64_t at = kHdr + kO1Bitmap + kO1Table * (uint64_t)t;
                    if (L < at + kO1Table) {
                        status = FQXV_RANS_E_TRUNCATED;
                        break;
                    }
                    status = load_table(at);
                    if (status != FQXV_RANS_OK) break;
                    uint8_t *C = T + kDecO1Base + kDecO1Ctx * (uint64_t)t;
                    uint16_t *S16 = reinterpret_cast<uint16_t *>(C);
                    uint32_t *FC = reinterpret_cast<uint32_t *>(C + kDecO1Slot);
                    if (tid < 256) FC[tid] = (sfreq[tid] << kScaleBits) | scum[tid];
                    for (int slot = tid; slot < (int)kTotFreq; slot += blockDim.x) {
                        int lo = 0, hi = 255;
                        while (lo < hi) {
                            const int mid = (lo + hi + 1) >> 1;
                            if (scum[mid] <= (uint32_t)slot) lo = mid; else hi = mid - 1;
                        }
                        S16[slot] = (uint16_t)(((uint32_t)lo << 8) | ctxmap[lo]);
                    }
                    __syncthreads();
                }
                hdr = kHdr + kO1Bitmap + kO1Table * (uint64_t)K;
                if (status == FQXV_RANS_OK && L < hdr + kStatesBytes) status = FQXV_RANS_E_TRUNCATED;
                if (status == FQXV_RANS_OK && n > S.dst_cap) status = FQXV_RANS_E_ALLOC;
                if (tid == 0) {
                    S.nctx = K;
                    S.ctx0 = ctxmap[0];
                }
            }
        }
        if (status == FQXV_RANS_OK && tid < kStates) S.states[tid] = ld_u32_le(p + hdr + 4 * tid);
        if (tid == 0) {
            // The renorm words follow the 32 states (scalar.rs:130-140).
            const uint64_t wbeg = hdr + kStatesBytes;
            S.status = status;
            S.words_off = S.src_off + wbeg;
            S.words_len = L > wbeg ? L - wbeg : 0;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ uint32_t load_word(const uint8_t *__restrict__ w, uint64_t j) {
    return (uint32_t)__ldg(w + 2 * j) | ((uint32_t)__ldg(w + 2 * j + 1) << 8);
}

// Renormalise the lanes in `need` (the reference's `while v < RANS_L`,
// scalar.rs:233-235). Fast path: every needing lane takes exactly one word,
// lane order = stream order. A lane whose value is 0 needs more than one word
// (only malformed streams do this); the round is then replayed lane by lane.
// Returns false on running out of words (scalar.rs:261, "truncated stream").
__device__ __forceinline__ bool renorm_round(uint32_t &v, bool need, const uint8_t *__restrict__ wb,
                                             uint64_t &wp, uint64_t navail, uint32_t lt) {
    const int lane = threadIdx.x & 31;
    const uint32_t cand = (wp + lane < navail) ? load_word(wb, wp + lane) : 0u;
    const uint32_t mask = __ballot_sync(0xffffffffu, need);
    if (__any_sync(0xffffffffu, need && v == 0)) {
        uint64_t wpl = wp;
        bool ok = true;
        for (int l = 0; l < 32; l++) {
            if (lane == l && need) {
                uint32_t vv = v;
                while (vv < kRansL) {
                    if (wpl >= navail) {
                        ok = false;
                        break;
                    }
                    vv = (vv << 16) | load_word(wb, wpl++);
                }
                v = vv;
            }
            wpl = __shfl_sync(0xffffffffu, wpl, l);
            ok = __shfl_sync(0xffffffffu, ok, l);
            if (!ok) return false;
        }
        wp = wpl;
        return true;
    }
    const uint32_t k = __popc(mask);
    if (wp + k > navail) return false;
    const uint32_t w = __shfl_sync(0xffffffffu, cand, __popc(mask & lt) & 31);
    if (need) v = (v << 16) | w;
    wp += k;
    return true;
}

// scalar.rs:157-178 / avx512.rs:78-134: order-0 decode of one stream.
__device__ __forceinline__ int decode_o0(const DecStream &S, const uint32_t *__restrict__ P,
                                         const uint8_t *__restrict__ src, uint8_t *__restrict__ out) {
    const int lane = threadIdx.x & 31;
    const uint32_t lt = lanemask_lt();
    const uint64_t n = S.n;
    uint32_t x = S.states[lane];
    const uint8_t *wb = src + S.words_off;
    const uint64_t navail = S.words_len / 2;
    uint64_t wp = 0;
    const uint64_t R = (n + 31) / 32;
    for (uint64_t r = 0; r < R; r++) {
        const uint64_t i = r * 32 + lane;
        const bool active = i < n;
        if ((r & 7) == 0 && lane == 0 && wp + 512 < navail)
            asm volatile("prefetch.global.L1 [%0];" ::"l"(wb + 2 * (wp + 512)));
        const uint32_t e = __ldg(P + (x & (kTotFreq - 1)));
        uint32_t v = ((e >> 20) + 1) * (x >> kScaleBits) + ((e >> 8) & 0xfffu);
        const bool need = active && v < kRansL;
        if (!renorm_round(v, need, wb, wp, navail, lt)) return FQXV_RANS_E_TRUNCATED;
        if (active) {
            out[i] = (uint8_t)e;
            x = v;
        }
    }
    return FQXV_RANS_OK;
}

// scalar.rs:180-217: order-1 decode. Each round resolves the context chain
// s_i = slot2sym[s_{i-1}][slot_i] lane by lane (the table lookups of a round
// are dependent), then all lanes advance their states together.
__device__ __forceinline__ int decode_o1(const DecStream &S, const uint8_t *__restrict__ T,
                                         const uint8_t *__restrict__ src, uint8_t *__restrict__ out) {
    const int lane = threadIdx.x & 31;
    const uint32_t lt = lanemask_lt();
    const uint64_t n = S.n;
    uint32_t x = S.states[lane];
    const uint8_t *wb = src + S.words_off;
    const uint64_t navail = S.words_len / 2;
    const bool all_present = S.nctx == 256;
    const uint8_t *base = T + kDecO1Base;
    uint64_t wp = 0;
    uint32_t t = (uint32_t)S.ctx0;
    const uint64_t R = (n + 31) / 32;
    for (uint64_t r = 0; r < R; r++) {
        const uint64_t i = r * 32 + lane;
        const bool active = i < n;
        const uint64_t left = n - r * 32;
        const int jmax = left < 32 ? (int)left : 32;
        if ((r & 7) == 0 && lane == 0 && wp + 512 < navail)
            asm volatile("prefetch.global.L1 [%0];" ::"l"(wb + 2 * (wp + 512)));
        const uint32_t slot = x & (kTotFreq - 1);
        uint32_t my_t = 0, my_e = 0;
        int absent_at = 32;
#pragma unroll
        for (int j = 0; j < 32; j++) {
            const uint32_t sl = __shfl_sync(0xffffffffu, slot, j);
            if (j < jmax) {
                if (!all_present && t == 0xffu) {
                    absent_at = j;
                    break;
                }
                const uint32_t e16 = __ldg(reinterpret_cast<const uint16_t *>(base + kDecO1Ctx * t) + sl);
                if (lane == j) {
                    my_t = t;
                    my_e = e16;
                }
                t = e16 & 0xffu;
            }
        }
        const bool valid = active && lane < absent_at;
        uint32_t v = 0;
        if (valid) {
            const uint32_t sym = my_e >> 8;
            const uint32_t fc = __ldg(reinterpret_cast<const uint32_t *>(base + kDecO1Ctx * my_t + kDecO1Slot) + sym);
            v = (fc >> kScaleBits) * (x >> kScaleBits) + slot - (fc & (kTotFreq - 1));
        }
        const bool need = valid && v < kRansL;
        if (!renorm_round(v, need, wb, wp, navail, lt)) return FQXV_RANS_E_TRUNCATED;
        if (absent_at < jmax) return FQXV_RANS_E_ABSENT_CONTEXT;
        if (active) {
            out[i] = (uint8_t)(my_e >> 8);
            x = v;
        }
    }
    return FQXV_RANS_OK;
}

__global__ void __launch_bounds__(kDecWarpsPerCta * 32)
    dec_run_kernel(const uint8_t *__restrict__ src, DecStream *__restrict__ streams,
                   const uint32_t *__restrict__ order, int nstreams, const uint8_t *__restrict__ tbl,
                   uint8_t *__restrict__ dst, int *__restrict__ queue) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        int j = 0;
        if (lane == 0) j = atomicAdd(queue, 1);
        j = __shfl_sync(0xffffffffu, j, 0);
        if (j >= nstreams) return;
        DecStream &S = streams[order[j]];
        if (S.status != FQXV_RANS_OK || S.n == 0) continue;
        const uint8_t *T = tbl + S.tbl_off;
        uint8_t *out = dst + S.dst_off;
        const int st = S.order == 0 ? decode_o0(S, reinterpret_cast<const uint32_t *>(T), src, out)
                                    : decode_o1(S, T, src, out);
        if (lane == 0) S.status = st;
        __syncwarp();
    }
}

void launch_dec_parse(const uint8_t *src, DecStream *streams, int nstreams, uint8_t *tbl, int grid,
                      cudaStream_t s) {
    if (nstreams <= 0) return;
    dec_parse_kernel<<<grid, kParseThreads, 0, s>>>(src, streams, nstreams, tbl);
}

void launch_dec_run(const uint8_t *src, DecStream *streams, const uint32_t *order, int nstreams,
                    const uint8_t *tbl, uint8_t *dst, int *queue, int grid, cudaStream_t s) {
    if (nstreams <= 0) return;
    dec_run_kernel<<<grid, kDecWarpsPerCta * 32, 0, s>>>(src, streams, order, nstreams, tbl, dst, queue);
}

}  // namespace fqxv
