// Decode path of the B200 rANS Nx16 coder.
//
//   1. dec_parse_kernel  one CTA per stream: header checks in the reference's
//      order (lib.rs:226-231, scalar.rs:143-217, model.rs:160-205), then the
//      decode tables in the table arena:
//        order-0: one packed word per slot ((f-1)<<20 | offset<<8 | sym, the
//                 layout of avx2.rs:29-54);
//        order-1 dense: all contexts and symbols renumbered densely (|D| <= 47)
//                 so that one u8 lookup chain[ctx][slot] gives the next
//                 context, plus a (freq << 12 | cum) table per (ctx, sym);
//        order-1 global: the same idea with u16 entries for larger alphabets.
//   2. one decode kernel per class, one warp per CTA, streams taken from a
//      device queue largest first. Lane l owns state l; renorm words are
//      handed out in stream order by a ballot/popc prefix over the lanes that
//      need one, read from a shared-memory ring that the warp refills with
//      16-byte loads issued eight-plus rounds ahead. The stream's tables are
//      staged into shared memory with one TMA bulk copy (cp.async.bulk +
//      mbarrier, bounded wait).
//      Order-1 resolves each round's context chain s_i = table[s_{i-1}][slot_i]
//      in four segments of eight lanes: the first segment from the known
//      context, the other three for every possible incoming context at once,
//      then three dependent lookups pick the real paths (11 dependent shared
//      memory reads per round instead of 32).
// Malformed input never faults: every read of the stream is bounds checked
// and errors are reported per stream as the reference's Malformed kinds.
#include <algorithm>
#include <mutex>

#include "rans_common.cuh"
#include "rans_internal.cuh"

namespace fqxv {

// ---------------------------------------------------------------------------
// header parse and table build
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(kParseThreads)
    dec_parse_kernel(const uint8_t *__restrict__ src, DecStream *__restrict__ streams, int nstreams,
                     uint8_t *__restrict__ tbl) {
    __shared__ uint32_t sfreq[256];
    __shared__ uint32_t scum[257];
    __shared__ uint32_t wsum[kParseThreads / 32];
    __shared__ uint8_t ctxmap[256];   // raw context -> present-table index (0xFF absent)
    __shared__ uint8_t ctxlist[256];  // present-table index -> raw context
    __shared__ uint8_t dmap[256];     // raw byte -> dense index (0xFF not in D)
    __shared__ uint8_t symseen[256];
    __shared__ uint16_t s_col[kTotFreq];  // dense format: column index of every slot
    __shared__ uint32_t s_bnd[kTotFreq / 32];   // dense format: boundary bitmap over the slots
    __shared__ int s_k, s_nd, s_bad, s_ncol;
    __shared__ uint8_t s_badst[256];
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
            S.cls = kClsNone;
            S.nd = 0;
            S.start = 0;
            S.tbl_bytes = 0;
            S.tbl_bytes_planes = 0;
        }
        if (status != FQXV_RANS_OK || n == 0) {
            if (tid == 0) S.status = status;
            __syncthreads();
            continue;
        }
        uint8_t *T = tbl + S.tbl_off;
        // Read one 256-entry frequency table at byte offset `at` (in bounds)
        // into sfreq/scum and validate it (model.rs:160-174).
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
            // Running sums are monotone: "some prefix exceeds" == "total exceeds".
            return tot > kTotFreq ? FQXV_RANS_E_FREQ_EXCEEDS
                                  : (tot != kTotFreq ? FQXV_RANS_E_FREQ_SUM : FQXV_RANS_OK);
        };
        // Symbol of `slot` in the table held in sfreq/scum: the largest s with
        // cum[s] <= slot (which always has f[s] > 0 in a valid table).
        auto slot_sym = [&](uint32_t slot) -> int {
            int lo = 0, hi = 255;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (scum[mid] <= slot) lo = mid; else hi = mid - 1;
            }
            return lo;
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
                    const int s = slot_sym((uint32_t)slot);
                    P[slot] = ((sfreq[s] - 1) << 20) | (((uint32_t)slot - scum[s]) << 8) | (uint32_t)s;
                }
                if (tid == 0) {
                    S.cls = kClsO0;
                    S.tbl_bytes = 16384;
                    S.tbl_bytes_planes = 16384;
                }
            }
        } else if (L < kHdr + kO1Bitmap) {
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
                        ctxlist[base] = (uint8_t)ctx;
                        ctxmap[ctx] = (uint8_t)(base++);
                    } else {
                        ctxmap[ctx] = 0xff;
                    }
                }
                if (lane == 31) s_k = (int)base;
            }
            if (tid < 256) symseen[tid] = 0;
            if (tid == 0) s_bad = 1 << 30;
            __syncthreads();
            const int K = s_k;
            // Pass 1: every table checked, one warp per table; the first
            // failing table in ascending context order decides the error,
            // truncation or validity, as the reference's sequential reads
            // do (scalar.rs:186-194, model.rs:160-174).
            for (int t = warp; t < K; t += kParseThreads / 32) {
                const uint64_t at = kHdr + kO1Bitmap + kO1Table * (uint64_t)t;
                int st = FQXV_RANS_OK;
                if (L < at + kO1Table) {
                    st = FQXV_RANS_E_TRUNCATED;
                } else {
                    uint32_t tot = 0;
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        const uint32_t f = (uint32_t)p[at + 16 * lane + 2 * k] | ((uint32_t)p[at + 16 * lane + 2 * k + 1] << 8);
                        tot += f;
                        if (f) symseen[lane * 8 + k] = 1;
                    }
                    const uint64_t tt = warp_sum_u64(tot);
                    // running sums are monotone: "some prefix exceeds" == "total exceeds"
                    st = tt > kTotFreq ? FQXV_RANS_E_FREQ_EXCEEDS : (tt != kTotFreq ? FQXV_RANS_E_FREQ_SUM : FQXV_RANS_OK);
                }
                if (st != FQXV_RANS_OK && lane == 0) {
                    s_badst[t] = (uint8_t)st;
                    atomicMin(&s_bad, t);
                }
            }
            __syncthreads();
            if (s_bad < K) status = s_badst[s_bad];
            hdr = kHdr + kO1Bitmap + kO1Table * (uint64_t)K;
            if (status == FQXV_RANS_OK && L < hdr + kStatesBytes) status = FQXV_RANS_E_TRUNCATED;
            if (status == FQXV_RANS_OK && n > S.dst_cap) status = FQXV_RANS_E_ALLOC;
            if (status == FQXV_RANS_OK) {
                // D = present contexts plus every symbol of their tables.
                if (warp == 0) {
                    uint32_t flags = 0;
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        const int s = lane * 8 + k;
                        if (symseen[s] || ctxmap[s] != 0xff) flags |= 1u << k;
                    }
                    const uint32_t c = __popc(flags);
                    uint32_t base = warp_incl_scan(c) - c;
#pragma unroll
                    for (int k = 0; k < 8; k++) dmap[lane * 8 + k] = (flags >> k) & 1u ? (uint8_t)(base++) : 0xff;
                    if (lane == 31) s_nd = (int)base;
                }
                __syncthreads();
                const int nd = s_nd;
                // f and exclusive cum of the 8 symbols lane owns in table t
                auto read_row = [&](int t, uint32_t f[8], uint32_t cum[8]) {
                    const uint64_t at = kHdr + kO1Bitmap + kO1Table * (uint64_t)t;
                    uint32_t run = 0;
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        f[k] = (uint32_t)p[at + 16 * lane + 2 * k] | ((uint32_t)p[at + 16 * lane + 2 * k + 1] << 8);
                        cum[k] = run;
                        run += f[k];
                    }
                    const uint32_t base = warp_incl_scan(run) - run;
#pragma unroll
                    for (int k = 0; k < 8; k++) cum[k] += base;
                };
                bool dense = nd <= kDenseMax;
                if (dense) {
                    // Boundaries: every slot where a present symbol of some
                    // context starts (slot 0 always, so a column exists even
                    // without any table); the column of a slot is the number
                    // of boundaries at or below it, minus one.
                    if (tid < (int)(kTotFreq / 32)) s_bnd[tid] = tid == 0 ? 1u : 0u;
                    __syncthreads();
                    for (int t = warp; t < K; t += kParseThreads / 32) {
                        uint32_t f[8], cum[8];
                        read_row(t, f, cum);
#pragma unroll
                        for (int k = 0; k < 8; k++)
                            if (f[k]) atomicOr(&s_bnd[cum[k] >> 5], 1u << (cum[k] & 31));
                    }
                    __syncthreads();
                    const uint32_t w = tid < (int)(kTotFreq / 32) ? s_bnd[tid] : 0u;
                    const uint32_t c = __popc(w);
                    const uint32_t incl = warp_incl_scan(c);
                    if (lane == 31) wsum[warp] = incl;
                    __syncthreads();
                    if (tid < (int)(kTotFreq / 32)) {
                        uint32_t run = incl - c;
                        for (int q = 0; q < warp; q++) run += wsum[q];
                        for (int b = 0; b < 32; b++) {
                            run += (w >> b) & 1u;
                            s_col[tid * 32 + b] = (uint16_t)(run - 1);
                        }
                    }
                    if (tid == 0) {
                        uint32_t tot = 0;
                        for (int q = 0; q < kParseThreads / 32; q++) tot += wsum[q];
                        s_ncol = (int)tot;
                    }
                    __syncthreads();
                    dense = dense_build_bytes(nd, (uint32_t)s_ncol) <= kDenseImageMax;
                }
                if (dense) {
                    const uint32_t ncol = (uint32_t)s_ncol;
                    const int dead = nd;
                    const int stride = nd + 1;
                    const uint32_t cs = dense_col_stride(nd);
                    const bool packed = dense_packed(nd);
                    uint8_t *M8 = T;
                    uint32_t *MB = reinterpret_cast<uint32_t *>(T + kDenseMB);
                    uint32_t *FC = reinterpret_cast<uint32_t *>(T + kDenseM);
                    uint8_t *DS = T + kDenseM + dense_fc_bytes(nd);
                    // byte columns: the image itself, or (packed form) scratch
                    // after it from which the u64 columns are packed
                    uint8_t *COL = T + (packed ? dense_table_bytes(nd, ncol) : dense_col_off(nd));
                    // Every column entry starts DEAD (rows of contexts without
                    // a table, the DEAD row, padding); FC starts zeroed.
                    const uint32_t deadw = 0x01010101u * (uint32_t)dead;
                    for (uint32_t i = tid; i < ncol * cs / 4; i += blockDim.x)
                        reinterpret_cast<uint32_t *>(COL)[i] = deadw;
                    for (int i = tid; i < stride * stride; i += blockDim.x) FC[i] = 0;
                    for (int i = tid; i < (int)kTotFreq; i += blockDim.x)
                        M8[i] = (uint8_t)(s_col[i] - s_col[i & ~255]);
                    if (tid < (int)(kTotFreq / 256)) MB[tid] = packed ? s_col[tid * 256] : s_col[tid * 256] * cs;
                    if (tid < 256 && dmap[tid] != 0xff) DS[dmap[tid]] = (uint8_t)tid;
                    __syncthreads();
                    // One warp per present context: its FC row, and its row
                    // of every column -- the columns of a symbol's slot range
                    // [cum, cum + f) are s_col[cum] .. s_col[cum + f - 1].
                    for (int t = warp; t < K; t += kParseThreads / 32) {
                        const int dc = dmap[ctxlist[t]];
                        uint32_t f[8], cum[8];
                        read_row(t, f, cum);
#pragma unroll
                        for (int k = 0; k < 8; k++) {
                            const uint32_t sym = lane * 8 + k;
                            if (f[k]) FC[dc * stride + dmap[sym]] = (f[k] << kScaleBits) | cum[k];
                        }
#pragma unroll
                        for (int k = 0; k < 8; k++) {
                            uint32_t m = __ballot_sync(0xffffffffu, f[k] != 0);
                            while (m) {
                                const int src = __ffs(m) - 1;
                                m &= m - 1;
                                const uint32_t c0 = __shfl_sync(0xffffffffu, cum[k], src);
                                const uint32_t fk = __shfl_sync(0xffffffffu, f[k], src);
                                const uint8_t dv = dmap[src * 8 + k];
                                const uint32_t j1 = s_col[c0 + fk - 1];
                                for (uint32_t j = s_col[c0] + lane; j <= j1; j += 32) COL[j * cs + dc] = dv;
                            }
                        }
                    }
                    __syncthreads();
                    // bit planes of every column, when they fit beside the image
                    const bool planes = dense_planes(nd) &&
                                        dense_table_bytes(nd, ncol) + kPlaneStride * ncol <= kDenseImageMax;
                    if (planes) {
                        uint32_t *PL = reinterpret_cast<uint32_t *>(T + dense_table_bytes(nd, ncol));
                        for (uint32_t j = warp; j < ncol; j += kParseThreads / 32) {
                            const uint32_t v = COL[j * cs + lane];
                            uint32_t w = 0;
#pragma unroll
                            for (int b = 0; b < 5; b++) {
                                const uint32_t pl = __ballot_sync(0xffffffffu, (v >> b) & 1u);
                                if (lane == b) w = __funnelshift_l(pl, pl, b);
                            }
                            if (lane < 8) PL[j * (kPlaneStride / 4) + lane] = w;
                        }
                        __syncthreads();
                    }
                    if (packed) {
                        // 16 entries of a 16-byte column -> 16 nibbles
                        uint64_t *PK = reinterpret_cast<uint64_t *>(T + dense_col_off(nd));
                        for (uint32_t j = tid; j < ncol; j += blockDim.x) {
                            uint64_t v = 0;
                            for (int d = 0; d < 16; d++) v |= (uint64_t)(COL[j * cs + d] & 15u) << (4 * d);
                            PK[j] = v;
                        }
                        __syncthreads();
                    }
                    if (tid == 0) {
                        S.cls = kClsO1Dense;
                        S.nd = nd;
                        S.start = dmap[0] != 0xff ? dmap[0] : dead;
                        S.tbl_bytes = dense_table_bytes(nd, ncol);
                        S.tbl_bytes_planes = S.tbl_bytes + (planes ? kPlaneStride * ncol : 0u);
                    }
                } else {
                    if (tid < 256) T[kDecCtxMap + tid] = ctxmap[tid];
                    for (int t = 0; t < K; t++) {
                        load_table(kHdr + kO1Bitmap + kO1Table * (uint64_t)t);
                        uint8_t *C = T + kDecO1Base + kDecO1Ctx * (uint64_t)t;
                        uint16_t *S16 = reinterpret_cast<uint16_t *>(C);
                        uint32_t *FCg = reinterpret_cast<uint32_t *>(C + kDecO1Slot);
                        if (tid < 256) FCg[tid] = (sfreq[tid] << kScaleBits) | scum[tid];
                        for (int slot = tid; slot < (int)kTotFreq; slot += blockDim.x) {
                            const int s = slot_sym((uint32_t)slot);
                            S16[slot] = (uint16_t)(((uint32_t)s << 8) | ctxmap[s]);
                        }
                        __syncthreads();
                    }
                    if (tid == 0) {
                        S.cls = kClsO1Global;
                        S.nd = nd;
                        S.ctx0 = ctxmap[0];
                    }
                }
                if (tid == 0) S.nctx = K;
            }
        }
        if (status == FQXV_RANS_OK && tid < kStates) S.states[tid] = ld_u32_le(p + hdr + 4 * tid);
        if (tid == 0) {
            // The renorm words follow the 32 states (scalar.rs:130-140).
            const uint64_t wbeg = hdr + kStatesBytes;
            S.status = status;
            if (status != FQXV_RANS_OK) S.cls = kClsNone;
            S.words_off = S.src_off + wbeg;
            S.words_len = L > wbeg ? L - wbeg : 0;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// shared pieces of the decode kernels
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint32_t load_word(const uint8_t *__restrict__ w, uint64_t j) {
    return (uint32_t)__ldg(w + 2 * j) | ((uint32_t)__ldg(w + 2 * j + 1) << 8);
}

// TMA bulk copy of a table image into shared memory, completion tracked by an
// mbarrier; the wait is bounded and reports failure instead of hanging.
struct TableStager {
    uint64_t *bar;
    uint32_t phase;

    __device__ void init(uint64_t *b) {
        bar = b;
        phase = 0;
        if ((threadIdx.x & 31) == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncwarp();
    }
    // bytes and both addresses are multiples of 16.
    __device__ void issue(void *dst, const void *src, uint32_t bytes) {
        __syncwarp();
        if ((threadIdx.x & 31) == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                         "r"(bytes)
                         : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_u32(dst)),
                "l"(src), "r"(bytes), "r"(smem_u32(bar))
                : "memory");
        }
    }
    // Polls the barrier's current phase at most `polls` times. The phase
    // advances only when the copy has landed, so a wait that gave up can be
    // followed by drain() on the same phase.
    __device__ bool wait(uint32_t polls) {
        uint32_t done = 0;
        for (uint32_t it = 0; it < polls && !done; it++) {
            asm volatile(
                "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                : "=r"(done)
                : "r"(smem_u32(bar)), "r"(phase)
                : "memory");
        }
        __syncwarp();
        const bool ok = __all_sync(0xffffffffu, done != 0);
        if (ok) phase ^= 1u;
        return ok;
    }
    // After a wait that gave up: wait for the same copy with the full bound,
    // so that it lands before its shared memory is reused or the CTA exits.
    // False when it still has not landed; the CTA must then issue no further
    // copy through this barrier (its phase is unknown).
    __device__ bool drain() { return wait(kWaitPolls); }
};

// Every job a CTA pops after its stager failed to drain reports a timeout
// without touching shared memory, so no stream of the batch is left without
// a status.
__device__ __forceinline__ void mark_timeout(DecStream &S) {
    if ((threadIdx.x & 31) == 0) S.status = FQXV_RANS_E_TIMEOUT;
    __syncwarp();
}

// Renorm-word ring: 4 segments of 512 bytes of the word region (16-byte
// aligned chunks, so a segment is one 16-byte load per lane). Segment q holds
// bytes [abase + 512 q, +512). Three segments are resident and a fourth is in
// flight in registers; it is stored when the read position enters the
// segment after the oldest, i.e. more than eight rounds before it is needed.
struct WordRing {
    const uint8_t *abase;   // 16-byte aligned start, <= first word byte
    const uint8_t *words;   // first word byte
    uint64_t avail;         // bytes from abase to the end of the region
    uint32_t lead;          // words - abase
    uint64_t next_seg;      // next segment to store
    uint4 pend;             // this lane's 16 bytes of segment next_seg
    uint8_t *ring;

    __device__ __forceinline__ uint4 fetch(uint64_t q) const {
        const uint64_t rel = 512 * q + 16 * (threadIdx.x & 31);
        if (rel < avail) return __ldg(reinterpret_cast<const uint4 *>(abase + rel));
        return make_uint4(0, 0, 0, 0);
    }
    __device__ __forceinline__ void put(uint64_t q, uint4 v) {
        *reinterpret_cast<uint4 *>(ring + ((512 * q + 16 * (threadIdx.x & 31)) & (kRingBytes - 1))) = v;
    }
    __device__ void reset(uint64_t q0) {
        __syncwarp();
        const uint4 a = fetch(q0), b = fetch(q0 + 1), c = fetch(q0 + 2);
        pend = fetch(q0 + 3);
        put(q0, a);
        put(q0 + 1, b);
        put(q0 + 2, c);
        next_seg = q0 + 3;
        __syncwarp();
    }
    __device__ void init(const uint8_t *w, uint64_t len, uint8_t *r) {
        words = w;
        abase = reinterpret_cast<const uint8_t *>((uintptr_t)w & ~(uintptr_t)15);
        lead = (uint32_t)(w - abase);
        avail = lead + len;
        ring = r;
        reset(0);
    }
    // Keep [pos, pos + 64) resident for the word index wp (warp-uniform).
    __device__ __forceinline__ void advance(uint64_t wp) {
        const uint64_t pos = lead + 2 * wp;
        while (pos >= 512 * (next_seg - 3)) {
            if (pos >= 512 * (next_seg - 2)) {
                reset(pos / 512);  // a jump of more than one segment
                return;
            }
            __syncwarp();
            put(next_seg, pend);
            next_seg++;
            pend = fetch(next_seg);
            __syncwarp();
        }
    }
    // Byte `rel` (relative to the word region) from the ring.
    __device__ __forceinline__ uint32_t byte(uint32_t rel) const { return ring[(lead + rel) & (kRingBytes - 1)]; }
    // Word j of the region; only the low bits of j matter (the ring is a
    // power-of-two window), so 32-bit arithmetic is exact here.
    __device__ __forceinline__ uint32_t word(uint32_t j) const {
        const uint32_t rel = lead + 2u * j;
        return (uint32_t)ring[rel & (kRingBytes - 1)] | ((uint32_t)ring[(rel + 1) & (kRingBytes - 1)] << 8);
    }
};

// Renormalise the lanes in `need` (the reference's `while v < RANS_L`,
// scalar.rs:233-235). Fast path: every needing lane takes exactly one word,
// lane order = stream order, from the ring. A lane whose value is 0 needs more
// than one word (only malformed streams do this); the round is then replayed
// lane by lane from global memory. Returns false when the words run out
// (scalar.rs:261, "truncated stream").
// `first` is set for the first round only: a state read from the header may
// be below 2^16, but every state a step produces is at least 2^16, after
// which v = f (x >> 12) + offset >= 16 and one word always suffices.
__device__ __forceinline__ bool renorm_round(uint32_t &v, bool need, const WordRing &R, uint64_t &wp,
                                             uint64_t navail, uint32_t lt, bool first = true) {
    const int lane = threadIdx.x & 31;
    const uint32_t cand = (wp + lane < navail) ? R.word((uint32_t)(wp + lane)) : 0u;
    const uint32_t mask = __ballot_sync(0xffffffffu, need);
    if (first && __any_sync(0xffffffffu, need && v == 0)) {
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
                    vv = (vv << 16) | load_word(R.words, wpl++);
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

__device__ __forceinline__ int pop_job(int *queue) {
    int j = 0;
    if ((threadIdx.x & 31) == 0) j = atomicAdd(queue, 1);
    return __shfl_sync(0xffffffffu, j, 0);
}

// ---------------------------------------------------------------------------
// order-0 (scalar.rs:157-178, avx512.rs:78-134)
// ---------------------------------------------------------------------------

// One decode round through the general path: any lane may need several
// words (states below 2^16 only come from a malformed header, so only the
// first round can see them), lanes past n idle, and running out of words is
// reported. Returns false on truncation.
__device__ __forceinline__ bool o0_general_round(uint32_t &x, const uint32_t *__restrict__ P, uint64_t r,
                                                 uint64_t n, WordRing &R, uint64_t &wp, uint64_t navail,
                                                 uint8_t *__restrict__ out, uint32_t lt) {
    const int lane = threadIdx.x & 31;
    R.advance(wp);
    const uint64_t i = r * 32 + lane;
    const bool active = i < n;
    const uint32_t e = P[x & (kTotFreq - 1)];
    uint32_t v = ((e >> 20) + 1) * (x >> kScaleBits) + ((e >> 8) & 0xfffu);
    const bool need = active && v < kRansL;
    if (!renorm_round(v, need, R, wp, navail, lt)) return false;
    if (active) {
        out[i] = (uint8_t)e;
        x = v;
    }
    return true;
}

// Copy of a decoded stream's output to the mirror (the device alias of a
// pinned host destination), made by the CTA that decoded it as soon as it is
// done: while other streams still decode, the host link takes the stream in
// 16-byte stores instead of the kernels' one-byte-per-lane output stores.
// `src` and `dst` are congruent modulo 16 (the host code places the device
// staging buffer so); the output was written by this CTA before the barrier
// that precedes the call, so plain loads see it.
__device__ __forceinline__ void mirror_out(const uint8_t *src, uint8_t *dst, uint64_t n, int t, int nt) {
    const uint64_t head = min(n, (uint64_t)((16u - ((uint32_t)(uintptr_t)dst & 15u)) & 15u));
    for (uint64_t i = t; i < head; i += nt) dst[i] = src[i];
    const uint64_t body = (n - head) / 16;
    const uint4 *s4 = reinterpret_cast<const uint4 *>(src + head);
    uint4 *d4 = reinterpret_cast<uint4 *>(dst + head);
    // eight loads in flight per thread before their stores: one load, then
    // its store, runs at the load's latency (about 1 GB/s for a warp over the
    // host link, measured on B200)
    uint64_t i = t;
    for (; i + 7 * (uint64_t)nt < body; i += 8 * (uint64_t)nt) {
        uint4 v[8];
#pragma unroll
        for (int k = 0; k < 8; k++) v[k] = s4[i + k * (uint64_t)nt];
#pragma unroll
        for (int k = 0; k < 8; k++) d4[i + k * (uint64_t)nt] = v[k];
    }
    for (; i < body; i += nt) d4[i] = s4[i];
    for (uint64_t i = head + 16 * body + t; i < n; i += nt) dst[i] = src[i];
}

__global__ void __launch_bounds__(32)
    dec_o0_kernel(const uint8_t *__restrict__ src, DecStream *__restrict__ streams,
                  const uint32_t *__restrict__ list, int nlist, const uint8_t *__restrict__ tbl,
                  uint8_t *__restrict__ dst, int *__restrict__ queue, uint32_t first_polls,
                  uint8_t *__restrict__ mirror) {
    extern __shared__ __align__(128) uint8_t sm[];
    __shared__ __align__(8) uint64_t bar;
    const int lane = threadIdx.x;
    const uint32_t lt = lanemask_lt();
    uint32_t *P = reinterpret_cast<uint32_t *>(sm);
    TableStager st;
    st.init(&bar);
    bool stuck = false;
    for (;;) {
        const int j = pop_job(queue);
        if (j >= nlist) return;
        DecStream &S = streams[list[j]];
        if (stuck) {
            mark_timeout(S);
            continue;
        }
        st.issue(P, tbl + S.tbl_off, 16384);
        WordRing R;
        R.init(src + S.words_off, S.words_len, sm + 16384);
        if (!st.wait(first_polls)) {
            stuck = !st.drain();
            mark_timeout(S);
            continue;
        }
        const uint64_t n = S.n;
        const uint64_t navail = S.words_len / 2;
        uint32_t x = S.states[lane];
        uint8_t *out = dst + S.dst_off;
        uint64_t wp = 0;
        int status = FQXV_RANS_OK;
        const uint64_t rounds = (n + 31) / 32, full = n / 32;
        // Fast-path window: W = word wp + lane, PE = the table entry that
        // word selects as the next slot. A lane that renormalises takes word
        // and next entry through one shuffle each from lane popc(earlier
        // needs), so the table lookup is off the round's critical path. The
        // next window's bytes are loaded as soon as the round's vote is
        // known and combined after its shuffles (a warp issues in order).
        uint32_t W = 0, PE = 0, e = 0;
        bool window = false;
        uint64_t r = 0;
        if (rounds && !o0_general_round(x, P, 0, n, R, wp, navail, out, lt)) status = FQXV_RANS_E_TRUNCATED;
        r = 1;
        constexpr int G = 8;  // rounds per branch-free group
        while (status == FQXV_RANS_OK && r < rounds) {
            // A group of G full rounds takes at most 32 G words and its window
            // reads 32 ahead, so it cannot run out of words or ring.
            if (r + G > full || wp + 32 * G + 64 > navail) {
                if (!o0_general_round(x, P, r, n, R, wp, navail, out, lt)) status = FQXV_RANS_E_TRUNCATED;
                r++;
                window = false;
                continue;
            }
            R.advance(wp);
            uint32_t w32 = (uint32_t)wp;
            if (!window) {
                W = R.word(w32 + lane);
                PE = P[W & (kTotFreq - 1)];
                e = P[x & (kTotFreq - 1)];
                window = true;
            }
            uint8_t *op = out + r * 32 + lane;
#pragma unroll
            for (int g = 0; g < G; g++) {
                const uint32_t v = ((e >> 20) + 1) * (x >> kScaleBits) + ((e >> 8) & 0xfffu);
                const uint32_t ev = P[v & (kTotFreq - 1)];
                const bool need = v < kRansL;
                const uint32_t mask = __ballot_sync(0xffffffffu, need);
                const uint32_t srcl = __popc(mask & lt);
                w32 += __popc(mask);
                const uint32_t b0 = R.byte(2 * (w32 + lane)), b1 = R.byte(2 * (w32 + lane) + 1);
                const uint32_t w = __shfl_sync(0xffffffffu, W, srcl);
                const uint32_t pe = __shfl_sync(0xffffffffu, PE, srcl);
                op[32 * g] = (uint8_t)e;
                x = need ? (v << 16) | w : v;
                e = need ? pe : ev;
                W = b0 | (b1 << 8);
                PE = P[W & (kTotFreq - 1)];
            }
            wp += (uint32_t)(w32 - (uint32_t)wp);
            r += G;
        }
        if (lane == 0) S.status = status;
        __syncwarp();
        if (mirror && status == FQXV_RANS_OK) mirror_out(out, mirror + S.dst_off, S.n, lane, 32);
    }
}

// ---------------------------------------------------------------------------
// order-1, dense tables in shared memory (scalar.rs:180-217)
// ---------------------------------------------------------------------------

// Decode one order-1 stream whose dense tables are in shared memory, with
// four warps (kO1Warps) per stream.
//
// Per round, the context chain d_i = col(slot_i)[d_{i-1}] of the 32 lanes is
// resolved in four segments of eight: segment 0 from the known incoming
// context, segments 1-3 for every possible incoming context at once, then
// three dependent lookups pick the real rows. A lane turns its slot into the
// byte offset of the slot's column once per round (one lookup in M), so each
// chain step is one byte load from a column: the steps of all chains of a
// segment read the same column (at most 48 bytes), not a row per context. Every warp holds its own copy
// of the 32 states, the word position and the incoming context, and runs the
// same renormalisation on the same words (from its own word ring), so the
// copies never diverge and one barrier per round suffices: each thread runs
// its share of the 3 nd speculative chains (TPL per thread, a template
// parameter) plus, on lane 0 of every warp, segment 0; the rows go to a
// double-buffered shared array, and after the barrier every warp resolves
// the round itself. Only warp 0 stores the output.
constexpr int kO1Warps = 4;
constexpr int kO1Threads = 32 * kO1Warps;
constexpr int kO1Workers = kO1Threads - kO1Warps;  // threads that run speculative chains

__device__ __forceinline__ void named_bar(int id) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(kO1Threads) : "memory");
}

// A slot's column, as the chains of a round need it: byte columns give the
// column's byte offset from the column base (a chain step is then one byte
// load); packed columns give the column itself, 16 four-bit entries in a
// u64 (a chain step is then a shift of a register).
struct ByteCols {
    const uint8_t *M8;
    const uint32_t *MB;
    uint32_t cs;  // column stride, bytes
    using T = uint32_t;
    __device__ __forceinline__ T operator()(uint32_t slot) const { return MB[slot >> 8] + (uint32_t)M8[slot] * cs; }
};
struct PackedCols {
    const uint8_t *M8;
    const uint32_t *MB;
    const uint64_t *PK;
    using T = uint64_t;
    __device__ __forceinline__ T operator()(uint32_t slot) const { return PK[MB[slot >> 8] + (uint32_t)M8[slot]]; }
};

// The rounds of one order-1 dense stream (scalar.rs:202-215), shared by the
// 4-warp and the 1-warp decoders: `resolve(slot, col, d, ctx)` runs one
// round's context chain from every lane's column (`Col`: byte or packed
// columns) and gives this lane's symbol and context; `store` says whether
// this warp writes the output.
//
// Rounds that cannot run out of words (and are not the first or the partial
// last round) take a branch-free fast path: the ring advances by predication,
// and a context without a table is only recorded, then reported once per
// run of fast rounds -- such a stream fails anyway, and a truncation cannot
// come earlier inside those rounds. Other rounds take the careful path with
// every check of scalar.rs:202-215 in order.
//
// `resolve` gets the lane's slot and its column. In fast rounds the next
// round's column is found while this round renormalises: a lane that takes a word gets its
// column with it (the column of every candidate word is looked up when the
// window is read, and shuffled along with the word); a lane that takes none
// looks up the column of its new value while the vote runs. So the M lookup
// is off the chain from one round to the next.
template <class Col, class Resolve>
__device__ __forceinline__ int o1_rounds(DecStream &S, WordRing &R, uint8_t *__restrict__ out, uint32_t lt,
                                         const Col &C, const uint32_t *__restrict__ FC,
                                         const uint8_t *__restrict__ DS, uint32_t stride, uint32_t dead, bool store,
                                         uint32_t x, Resolve &&resolve) {
    using CT = typename Col::T;
    const int lane = threadIdx.x & 31;
    const uint64_t n = S.n;
    const uint64_t navail = S.words_len / 2;
    uint64_t wp = 0;
    const uint64_t rounds = (n + 31) / 32, full = n / 32;
    uint64_t r = 0;
    int status = FQXV_RANS_OK;
    while (r < rounds && status == FQXV_RANS_OK) {
        const int64_t spare = (int64_t)navail - (int64_t)wp - 64;
        int64_t cnt = spare > 0 ? spare / 32 : 0;
        const int64_t left_full = r < full ? (int64_t)(full - r) : 0;
        if (cnt > left_full) cnt = left_full;
        if (r == 0 || cnt <= 0) {
            // careful round (scalar.rs:202-215 in order)
            R.advance(wp);
            const uint64_t i = r * 32 + lane;
            const bool active = i < n;
            const uint32_t slot = x & (kTotFreq - 1);
            uint32_t d, ctx;
            resolve(slot, C(slot), d, ctx);
            const uint32_t deadmask = __ballot_sync(0xffffffffu, active && d == dead);
            const int absent_at = deadmask ? __ffs(deadmask) - 1 : 32;
            const bool valid = active && lane < absent_at;
            const uint32_t fc = FC[ctx * stride + d];
            uint32_t v = (fc >> kScaleBits) * (x >> kScaleBits) + slot - (fc & (kTotFreq - 1));
            const bool need = valid && v < kRansL;
            if (!renorm_round(v, need, R, wp, navail, lt, r == 0)) {
                status = FQXV_RANS_E_TRUNCATED;
                break;
            }
            if (absent_at < 32) {
                status = FQXV_RANS_E_ABSENT_CONTEXT;
                break;
            }
            if (active) {
                if (store) out[i] = DS[d];
                x = v;
            }
            r++;
            continue;
        }
        // fast rounds: each takes at most 32 words, cnt of them fit.
        R.advance(wp);
        uint32_t w32 = (uint32_t)wp;
        uint32_t adv_at = (uint32_t)((512u * (uint32_t)(R.next_seg - 3) - R.lead + 1u) / 2u);
        uint32_t sawdead = 0;
        uint8_t *op = out + r * 32 + lane;
        CT cb = C(x & (kTotFreq - 1));
        for (int64_t c = 0; c < cnt; c++) {
            // predicated one-segment ring advance (a round moves <= 64 bytes)
            const bool adv = w32 - (uint32_t)wp >= adv_at - (uint32_t)wp;
            if (adv) {
                R.put(R.next_seg, R.pend);
                R.next_seg++;
                R.pend = R.fetch(R.next_seg);
                adv_at += 256u;
            }
            __syncwarp();
            const uint32_t cand = R.word(w32 + lane);
            const CT cbc = C(cand & (kTotFreq - 1));
            const uint32_t slot = x & (kTotFreq - 1);
            uint32_t d, ctx;
            resolve(slot, cb, d, ctx);
            sawdead |= d == dead;
            const uint32_t fc = FC[ctx * stride + d];
            const uint32_t v = (fc >> kScaleBits) * (x >> kScaleBits) + slot - (fc & (kTotFreq - 1));
            const CT cbv = C(v & (kTotFreq - 1));
            const bool need = v < kRansL;
            const uint32_t mask = __ballot_sync(0xffffffffu, need);
            const uint32_t srcl = __popc(mask & lt) & 31;
            const uint32_t w = __shfl_sync(0xffffffffu, cand, srcl);
            const CT cbw = __shfl_sync(0xffffffffu, cbc, srcl);
            if (store) *op = DS[d];
            op += 32;
            x = need ? (v << 16) | w : v;
            cb = need ? cbw : cbv;
            w32 += __popc(mask);
        }
        wp += (uint32_t)(w32 - (uint32_t)wp);
        r += (uint64_t)cnt;
        if (__any_sync(0xffffffffu, sawdead != 0)) status = FQXV_RANS_E_ABSENT_CONTEXT;
    }
    return status;
}

// Rows of the speculative chains, 16 bytes each: the eight chain values
// (d_0 the top byte of .x, d_7 the low byte of .y) and, in .z, the byte
// offset of the row the next segment continues from (the DEAD row when the
// chain ends in a context without a table), so that resolving a round is
// three dependent loads and no index arithmetic. Row kDeadRow repeats DEAD;
// row kPadRow takes the stores of threads without a task.
constexpr uint32_t kDeadRow = 3 * kDenseMax;
constexpr uint32_t kPadRow = kDeadRow + 1;
static_assert(kPadRow <= kOutRows, "row array too small");

// The parts of a dense table image in shared memory.
struct DenseImage {
    const uint8_t *M8;     // slot -> column, less its 256-slot block's first column
    const uint32_t *MB;    // per 256-slot block: its first column (byte offset for byte columns)
    const uint8_t *COL;    // columns
    const uint32_t *FC;    // (freq << 12) | cum per (context, symbol)
    const uint8_t *DS;     // dense index -> byte
    uint32_t stride;       // FC row stride (nd + 1)
    uint32_t dead;
    __device__ DenseImage(const uint8_t *sm, int nd)
        : M8(sm),
          MB(reinterpret_cast<const uint32_t *>(sm + kDenseMB)),
          COL(sm + dense_col_off(nd)),
          FC(reinterpret_cast<const uint32_t *>(sm + kDenseM)),
          DS(sm + kDenseM + dense_fc_bytes(nd)),
          stride((uint32_t)nd + 1),
          dead((uint32_t)nd) {}
};

template <int TPL>
__device__ __forceinline__ int o1d_stream(DecStream &S, const uint8_t *__restrict__ sm, WordRing &R,
                                          uint4 (*__restrict__ rows)[kOutRows + 1], uint8_t *__restrict__ out,
                                          uint32_t lt) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nd = S.nd;
    const DenseImage I(sm, nd);
    const uint32_t dead = I.dead;
    const int nspec = 3 * nd;
    // This thread's chains: lane 0 of each warp runs segment 0 (q = 0); the
    // other threads split the speculative tasks u = (seg - 1) nd + c.
    const int worker = warp * 31 + lane - 1;
    uint32_t seg_q[TPL], c_q[TPL], idx_q[TPL], nbase_q[TPL];
#pragma unroll
    for (int q = 0; q < TPL; q++) {
        const int u = worker + kO1Workers * q;
        const bool valid = lane != 0 && u < nspec;
        seg_q[q] = lane == 0 ? 0u : valid ? (uint32_t)(1 + u / nd) : 1u;
        c_q[q] = valid ? (uint32_t)(u % nd) : 0u;
        idx_q[q] = valid ? (uint32_t)u : kPadRow;
        nbase_q[q] = seg_q[q] * (uint32_t)nd;  // first row of the next segment
    }
    const uint8_t *COL = I.COL;
    const uint32_t deadw = 0x01010101u * dead;
    if (tid == 0) {
        rows[0][kDeadRow] = make_uint4(deadw, deadw, kDeadRow * 16u, 0u);
        rows[1][kDeadRow] = make_uint4(deadw, deadw, kDeadRow * 16u, 0u);
    }
    const uint32_t x = S.states[lane];
    uint32_t din = (uint32_t)S.start;
    const int seg = lane >> 3, pos = lane & 7;
    const uint32_t shd = 24u - 8u * (uint32_t)(pos & 3);        // byte pos of a row half
    const uint32_t shc = 24u - 8u * (uint32_t)((pos + 3) & 3);  // byte pos - 1
    uint32_t buf = 0;

    // One round: the chains of this thread, the barrier, then the resolved
    // symbol d and context ctx of this lane.
    auto resolve = [&](uint32_t, uint32_t cb, uint32_t &d, uint32_t &ctx) {
        uint4 mine[TPL];
#pragma unroll
        for (int q = 0; q < TPL; q++) {
            uint32_t sl[8];
#pragma unroll
            for (int k = 0; k < 8; k++) sl[k] = __shfl_sync(0xffffffffu, cb, 8 * seg_q[q] + k);
            uint32_t dd = (q == 0 && lane == 0) ? din : c_q[q];
            uint32_t hi = 0, lo = 0;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                dd = COL[sl[k] + dd];
                hi = hi * 256u + dd;
            }
#pragma unroll
            for (int k = 4; k < 8; k++) {
                dd = COL[sl[k] + dd];
                lo = lo * 256u + dd;
            }
            mine[q] = make_uint4(hi, lo, 16u * (dd == dead ? kDeadRow : nbase_q[q] + dd), 0u);
        }
        uint4 *rb = rows[buf];
#pragma unroll
        for (int q = 0; q < TPL; q++)
            if (q > 0 || lane != 0) rb[idx_q[q]] = mine[q];
        uint4 r0;
        r0.x = __shfl_sync(0xffffffffu, mine[0].x, 0);
        r0.y = __shfl_sync(0xffffffffu, mine[0].y, 0);
        r0.z = __shfl_sync(0xffffffffu, mine[0].z, 0);
        named_bar(1);
        const uint8_t *rbb = reinterpret_cast<const uint8_t *>(rb);
        const uint4 r1 = *reinterpret_cast<const uint4 *>(rbb + r0.z);
        const uint4 r2 = *reinterpret_cast<const uint4 *>(rbb + r1.z);
        const uint32_t rx = seg == 0 ? r0.x : seg == 1 ? r1.x : r2.x;
        const uint32_t ry = seg == 0 ? r0.y : seg == 1 ? r1.y : r2.y;
        const uint32_t ine = seg == 0 ? din : seg == 1 ? (r0.y & 0xffu) : (r1.y & 0xffu);
        const uint4 r3 = *reinterpret_cast<const uint4 *>(rbb + r2.z);
        const uint32_t row_x = seg == 3 ? r3.x : rx;
        const uint32_t row_y = seg == 3 ? r3.y : ry;
        const uint32_t in = seg == 3 ? (r2.y & 0xffu) : ine;
        d = ((pos < 4 ? row_x : row_y) >> shd) & 0xffu;
        ctx = pos == 0 ? in : ((pos <= 4 ? row_x : row_y) >> shc) & 0xffu;
        din = r3.y & 0xffu;
        buf ^= 1u;
    };

    return o1_rounds(S, R, out, lt, ByteCols{I.M8, I.MB, dense_col_stride(nd)}, I.FC, I.DS, I.stride, dead, warp == 0, x, resolve);
}

// Four-warp decode of a stream with bit-plane columns (kSmallMaxNd < |D| <=
// kPlaneMaxNd). Warp w >= 1 runs segment w for every incoming context, lane
// c from context c, and lane 31 of every warp runs segment 0 from the known
// context, so each warp has the first segment's row in registers. A chain
// step looks its next context up in the column's five bit planes (loaded
// into registers once per round): plane p rotated right by the context puts
// the entry's bit p at bit p, and four bit selects merge the five. Rows are
// (segment, context) pairs, 32 per segment; row (s, 31) is the DEAD row
// when |D| = 31 (the DEAD context is then 31, whose lane runs segment 0)
// and is never reached otherwise. The round is then resolved as in
// o1d_stream: three dependent row loads after the barrier.
__device__ __forceinline__ int o1p_stream(DecStream &S, const uint8_t *__restrict__ sm, WordRing &R,
                                          uint4 (*__restrict__ rows)[kOutRows + 1], uint8_t *__restrict__ out,
                                          uint32_t lt) {
    static_assert(4 * 32 <= kOutRows + 1, "row array holds four segments of 32 rows");
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nd = S.nd;
    const DenseImage I(sm, nd);
    const uint32_t dead = I.dead;
    const uint8_t *PL = sm + S.tbl_bytes;
    const uint32_t myseg = lane == 31 ? 0u : (uint32_t)warp;
    const bool writer = warp >= 1 && lane < 31;
    const uint32_t nbase = 32u * (myseg + 1u);  // row of context 0 in the next segment
    const uint32_t deadw = 0x01010101u * dead;
    if (tid < 6) {
        const uint32_t sg = 1u + (uint32_t)(tid % 3);
        rows[tid / 3][32u * sg + 31u] = make_uint4(deadw, deadw, 16u * (32u * (sg + 1u) + 31u), 0u);
    }
    uint32_t din = (uint32_t)S.start;
    const int seg = lane >> 3, pos = lane & 7;
    const uint32_t shd = 24u - 8u * (uint32_t)(pos & 3);
    const uint32_t shc = 24u - 8u * (uint32_t)((pos + 3) & 3);
    uint32_t buf = 0;

    auto resolve = [&](uint32_t, uint32_t cb, uint32_t &d, uint32_t &ctx) {
        uint32_t q[8][5];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const uint32_t off = __shfl_sync(0xffffffffu, cb, 8 * myseg + k);
            const uint4 a = *reinterpret_cast<const uint4 *>(PL + off);
            q[k][0] = a.x;
            q[k][1] = a.y;
            q[k][2] = a.z;
            q[k][3] = a.w;
            q[k][4] = *reinterpret_cast<const uint32_t *>(PL + off + 16);
        }
        uint32_t dd = lane == 31 ? din : (uint32_t)lane;
        uint32_t hi = 0, lo = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const uint32_t t0 = __funnelshift_r(q[k][0], q[k][0], dd);
            const uint32_t t1 = __funnelshift_r(q[k][1], q[k][1], dd);
            const uint32_t t2 = __funnelshift_r(q[k][2], q[k][2], dd);
            const uint32_t t3 = __funnelshift_r(q[k][3], q[k][3], dd);
            const uint32_t t4 = __funnelshift_r(q[k][4], q[k][4], dd);
            const uint32_t a = (t0 & 1u) | (t1 & ~1u);
            const uint32_t b = (t2 & 7u) | (t3 & ~7u);
            const uint32_t c = (a & 3u) | (b & ~3u);
            // bits above 4 are left over from the planes: a funnel shift
            // uses its amount mod 32, and the row keeps the clean value
            dd = (c & 15u) | (t4 & ~15u);
            if (k < 4) hi = (hi << 8) | (dd & 31u);
            else lo = (lo << 8) | (dd & 31u);
        }
        const uint32_t nx = 16u * (nbase + (dd & 31u));
        uint4 *rb = rows[buf];
        if (writer) rb[32 * warp + lane] = make_uint4(hi, lo, nx, 0u);
        uint4 r0;
        r0.x = __shfl_sync(0xffffffffu, hi, 31);
        r0.y = __shfl_sync(0xffffffffu, lo, 31);
        r0.z = __shfl_sync(0xffffffffu, nx, 31);
        named_bar(1);
        const uint8_t *rbb = reinterpret_cast<const uint8_t *>(rb);
        const uint4 r1 = *reinterpret_cast<const uint4 *>(rbb + r0.z);
        const uint4 r2 = *reinterpret_cast<const uint4 *>(rbb + r1.z);
        const uint32_t rx = seg == 0 ? r0.x : seg == 1 ? r1.x : r2.x;
        const uint32_t ry = seg == 0 ? r0.y : seg == 1 ? r1.y : r2.y;
        const uint32_t ine = seg == 0 ? din : seg == 1 ? (r0.y & 0xffu) : (r1.y & 0xffu);
        const uint4 r3 = *reinterpret_cast<const uint4 *>(rbb + r2.z);
        const uint32_t row_x = seg == 3 ? r3.x : rx;
        const uint32_t row_y = seg == 3 ? r3.y : ry;
        const uint32_t in = seg == 3 ? (r2.y & 0xffu) : ine;
        d = ((pos < 4 ? row_x : row_y) >> shd) & 0xffu;
        ctx = pos == 0 ? in : ((pos <= 4 ? row_x : row_y) >> shc) & 0xffu;
        din = r3.y & 0xffu;
        buf ^= 1u;
    };

    return o1_rounds(S, R, out, lt, ByteCols{I.M8, I.MB, dense_col_stride(nd)}, I.FC, I.DS, I.stride, dead, warp == 0, S.states[lane], resolve);
}

__global__ void __launch_bounds__(kO1Threads, 1)
    dec_o1d_kernel(const uint8_t *__restrict__ src, DecStream *__restrict__ streams,
                   const uint32_t *__restrict__ list, int nlist, const uint8_t *__restrict__ tbl,
                   uint8_t *__restrict__ dst, int *__restrict__ queue, uint32_t ring_off,
                   uint32_t first_polls, uint8_t *__restrict__ mirror) {
    extern __shared__ __align__(128) uint8_t sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ __align__(16) uint4 s_rows[2][kOutRows + 1];
    __shared__ int s_job, s_ok, s_stuck;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t lt = lanemask_lt();
    TableStager st;
    if (warp == 0) st.init(&bar);
    if (tid == 0) s_stuck = 0;
    __syncthreads();
    for (;;) {
        if (tid == 0) s_job = atomicAdd(queue, 1);
        __syncthreads();
        const int j = s_job;
        __syncthreads();
        if (j >= nlist) return;
        DecStream &S = streams[list[j]];
        if (warp == 0) {
            bool ok = false;
            if (!s_stuck) {
                st.issue(sm, tbl + S.tbl_off, S.tbl_bytes_planes);
                ok = st.wait(first_polls);
                if (!ok && !st.drain() && lane == 0) s_stuck = 1;
            }
            if (!ok) mark_timeout(S);
            if (lane == 0) s_ok = ok;
        }
        // every warp reads the words through its own ring
        WordRing R;
        R.init(src + S.words_off, S.words_len, sm + ring_off + warp * kRingBytes);
        __syncthreads();  // the table image is visible to every warp
        if (!s_ok) continue;
        uint8_t *out = dst + S.dst_off;
        const int tpl = (3 * S.nd + kO1Workers - 1) / kO1Workers;
        const int status = S.tbl_bytes_planes > S.tbl_bytes ? o1p_stream(S, sm, R, s_rows, out, lt)
                           : tpl <= 1                       ? o1d_stream<1>(S, sm, R, s_rows, out, lt)
                                                            : o1d_stream<2>(S, sm, R, s_rows, out, lt);
        if (tid == 0) S.status = status;
        __syncthreads();
        if (mirror && status == FQXV_RANS_OK) mirror_out(out, mirror + S.dst_off, S.n, tid, kO1Threads);
    }
}

// ---------------------------------------------------------------------------
// order-1, one warp per stream
// ---------------------------------------------------------------------------

// Alphabets of up to kShflMaxNd symbols: every chain fits in one warp:
// lane 0 runs segment 0 from the known context, lanes 1..3 nd run segment
// s >= 1 from every possible incoming context (lane 1 + (s - 1) nd + c),
// lane 31 holds the DEAD row. Each row carries the lane of the row the next
// segment continues from, so resolving a round is three dependent shuffles
// -- no shared rows, no barrier, no copies of the states. The columns are
// packed (16 four-bit entries per u64; for NARROW, |D| <= 7, the low 32 bits
// hold them all), so a chain step is a shift and a mask of a register
// instead of a shared-memory load.
template <bool NARROW>
__device__ __forceinline__ int o1s_stream(DecStream &S, const uint8_t *__restrict__ sm, WordRing &R,
                                          uint8_t *__restrict__ out, uint32_t lt) {
    const int lane = threadIdx.x & 31;
    const int nd = S.nd;
    const DenseImage I(sm, nd);
    const uint32_t dead = I.dead;
    const bool task = lane >= 1 && lane <= 3 * nd;
    const uint32_t myseg = task ? (uint32_t)(1 + (lane - 1) / nd) : 0u;
    const uint32_t myc = task ? (uint32_t)((lane - 1) % nd) : 0u;
    const uint32_t nbase = 1u + myseg * (uint32_t)nd;  // lane of the next segment's context-0 row
    const uint64_t *PK = reinterpret_cast<const uint64_t *>(I.COL);
    const uint32_t deadw = 0x01010101u * dead;
    uint32_t din = (uint32_t)S.start;
    const int seg = lane >> 3, pos = lane & 7;
    const uint32_t shd = 24u - 8u * (uint32_t)(pos & 3);
    const uint32_t shc = 24u - 8u * (uint32_t)((pos + 3) & 3);

    auto resolve = [&](uint32_t, uint64_t col, uint32_t &d, uint32_t &ctx) {
        uint32_t dd = lane == 0 ? din : myc;
        uint32_t hi = 0, lo = 0;
        if constexpr (NARROW) {
            uint32_t sl[8];
            const uint32_t c32 = (uint32_t)col;
#pragma unroll
            for (int k = 0; k < 8; k++) sl[k] = __shfl_sync(0xffffffffu, c32, 8 * myseg + k);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                dd = (sl[k] >> (dd << 2)) & 15u;
                hi = (hi << 8) | dd;
            }
#pragma unroll
            for (int k = 4; k < 8; k++) {
                dd = (sl[k] >> (dd << 2)) & 15u;
                lo = (lo << 8) | dd;
            }
        } else {
            uint64_t sl[8];
#pragma unroll
            for (int k = 0; k < 8; k++) sl[k] = __shfl_sync(0xffffffffu, col, 8 * myseg + k);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                dd = (uint32_t)(sl[k] >> (dd << 2)) & 15u;
                hi = (hi << 8) | dd;
            }
#pragma unroll
            for (int k = 4; k < 8; k++) {
                dd = (uint32_t)(sl[k] >> (dd << 2)) & 15u;
                lo = (lo << 8) | dd;
            }
        }
        uint32_t nx = dd == dead ? 31u : nbase + dd;
        if (lane == 31) {
            hi = deadw;
            lo = deadw;
            nx = 31u;
        }
        // Three levels of shuffles: every lane first learns the row two
        // segments on (nn, the next of its next); then lane 0's row gives
        // the rows of segments 1 and 2 at once (n0, and n1 = nn of lane 0),
        // and those give the rows of segments 2 and 3 (n2 = nn of lane n0).
        const uint32_t nn = __shfl_sync(0xffffffffu, nx, nx);
        const uint32_t r0x = __shfl_sync(0xffffffffu, hi, 0), r0y = __shfl_sync(0xffffffffu, lo, 0);
        const uint32_t n0 = __shfl_sync(0xffffffffu, nx, 0);
        const uint32_t n1 = __shfl_sync(0xffffffffu, nn, 0);
        const uint32_t r1x = __shfl_sync(0xffffffffu, hi, n0), r1y = __shfl_sync(0xffffffffu, lo, n0);
        const uint32_t n2 = __shfl_sync(0xffffffffu, nn, n0);
        const uint32_t r2x = __shfl_sync(0xffffffffu, hi, n1), r2y = __shfl_sync(0xffffffffu, lo, n1);
        const uint32_t rx = seg == 0 ? r0x : seg == 1 ? r1x : r2x;
        const uint32_t ry = seg == 0 ? r0y : seg == 1 ? r1y : r2y;
        const uint32_t ine = seg == 0 ? din : seg == 1 ? (r0y & 0xffu) : (r1y & 0xffu);
        const uint32_t r3x = __shfl_sync(0xffffffffu, hi, n2), r3y = __shfl_sync(0xffffffffu, lo, n2);
        const uint32_t row_x = seg == 3 ? r3x : rx;
        const uint32_t row_y = seg == 3 ? r3y : ry;
        const uint32_t in = seg == 3 ? (r2y & 0xffu) : ine;
        d = ((pos < 4 ? row_x : row_y) >> shd) & 0xffu;
        ctx = pos == 0 ? in : ((pos <= 4 ? row_x : row_y) >> shc) & 0xffu;
        din = r3y & 0xffu;
    };
    return o1_rounds(S, R, out, lt, PackedCols{I.M8, I.MB, PK}, I.FC, I.DS, I.stride, dead, true, S.states[lane],
                     resolve);
}

// Wider alphabets in one warp: lane 0 runs segment 0; lanes 1-10, 11-20 and
// 21-30 run segments 1, 2 and 3, lane i of a segment following the incoming
// contexts i, i + 10, ... (TPL chains per lane, TPL = ceil(nd / 10),
// interleaved so their steps overlap). All chains of a lane share one
// segment, so a round needs eight column shuffles per lane whatever TPL is.
// Rows go to a double-buffered shared array (rows 0 .. 3 nd - 1, then the
// DEAD row and a row for lanes without a task) and are resolved after a
// __syncwarp with three dependent loads, as in the four-warp decoder, but
// without its barrier or its replicated states: one warp and ~30 KB of
// shared memory per full-range quality stream, so several streams share an
// SM. PACKED (|D| <= kSmallMaxNd) steps chains in registers on packed
// columns; otherwise a step is a byte load from a column.
constexpr int kWideLanes = 10;  // lanes per speculative segment

template <int TPL, bool PACKED>
__device__ __forceinline__ int o1w_stream(DecStream &S, const uint8_t *__restrict__ sm, WordRing &R,
                                          uint4 *__restrict__ rows0, uint4 *__restrict__ rows1,
                                          uint8_t *__restrict__ out, uint32_t lt) {
    const int lane = threadIdx.x & 31;
    const int nd = S.nd;
    const DenseImage I(sm, nd);
    const uint32_t dead = I.dead;
    const uint32_t deadrow = 3u * (uint32_t)nd, padrow = deadrow + 1u;
    const bool worker = lane >= 1 && lane <= 3 * kWideLanes;
    const uint32_t myseg = worker ? (uint32_t)(1 + (lane - 1) / kWideLanes) : 0u;
    const uint32_t li = worker ? (uint32_t)((lane - 1) % kWideLanes) : 0u;
    const uint32_t nbase = myseg * (uint32_t)nd;  // first row of the next segment
    uint32_t c_q[TPL], idx_q[TPL];
#pragma unroll
    for (int q = 0; q < TPL; q++) {
        const uint32_t c = li + kWideLanes * q;
        const bool valid = worker && c < (uint32_t)nd;
        c_q[q] = valid ? c : 0u;
        idx_q[q] = valid ? (myseg - 1) * (uint32_t)nd + c : padrow;
    }
    const uint8_t *COL = I.COL;
    const uint32_t deadw = 0x01010101u * dead;
    if (lane == 0) {
        rows0[deadrow] = make_uint4(deadw, deadw, deadrow * 16u, 0u);
        rows1[deadrow] = make_uint4(deadw, deadw, deadrow * 16u, 0u);
    }
    __syncwarp();
    uint32_t din = (uint32_t)S.start;
    const int seg = lane >> 3, pos = lane & 7;
    const uint32_t shd = 24u - 8u * (uint32_t)(pos & 3);
    const uint32_t shc = 24u - 8u * (uint32_t)((pos + 3) & 3);
    uint32_t buf = 0;

    auto resolve = [&](uint32_t, auto cb, uint32_t &d, uint32_t &ctx) {
        using CT = decltype(cb);
        CT sl[8];
#pragma unroll
        for (int k = 0; k < 8; k++) sl[k] = __shfl_sync(0xffffffffu, cb, 8 * myseg + k);
        uint32_t dd[TPL], hi[TPL], lo[TPL];
#pragma unroll
        for (int q = 0; q < TPL; q++) {
            dd[q] = (q == 0 && lane == 0) ? din : c_q[q];
            hi[q] = 0;
            lo[q] = 0;
        }
#pragma unroll
        for (int k = 0; k < 8; k++) {
#pragma unroll
            for (int q = 0; q < TPL; q++) {
                if constexpr (PACKED) dd[q] = (uint32_t)(sl[k] >> (dd[q] << 2)) & 15u;
                else dd[q] = COL[sl[k] + dd[q]];
                if (k < 4) hi[q] = (hi[q] << 8) | dd[q];
                else lo[q] = (lo[q] << 8) | dd[q];
            }
        }
        uint4 *rb = buf ? rows1 : rows0;
#pragma unroll
        for (int q = 0; q < TPL; q++) {
            const uint32_t nx = 16u * (dd[q] == dead ? deadrow : nbase + dd[q]);
            if (q > 0 || lane != 0) rb[idx_q[q]] = make_uint4(hi[q], lo[q], nx, 0u);
        }
        uint4 r0;
        r0.x = __shfl_sync(0xffffffffu, hi[0], 0);
        r0.y = __shfl_sync(0xffffffffu, lo[0], 0);
        r0.z = __shfl_sync(0xffffffffu, 16u * (dd[0] == dead ? deadrow : nbase + dd[0]), 0);
        __syncwarp();
        const uint8_t *rbb = reinterpret_cast<const uint8_t *>(rb);
        const uint4 r1 = *reinterpret_cast<const uint4 *>(rbb + r0.z);
        const uint4 r2 = *reinterpret_cast<const uint4 *>(rbb + r1.z);
        const uint32_t rx = seg == 0 ? r0.x : seg == 1 ? r1.x : r2.x;
        const uint32_t ry = seg == 0 ? r0.y : seg == 1 ? r1.y : r2.y;
        const uint32_t ine = seg == 0 ? din : seg == 1 ? (r0.y & 0xffu) : (r1.y & 0xffu);
        const uint4 r3 = *reinterpret_cast<const uint4 *>(rbb + r2.z);
        const uint32_t row_x = seg == 3 ? r3.x : rx;
        const uint32_t row_y = seg == 3 ? r3.y : ry;
        const uint32_t in = seg == 3 ? (r2.y & 0xffu) : ine;
        d = ((pos < 4 ? row_x : row_y) >> shd) & 0xffu;
        ctx = pos == 0 ? in : ((pos <= 4 ? row_x : row_y) >> shc) & 0xffu;
        din = r3.y & 0xffu;
        buf ^= 1u;
    };
    if constexpr (PACKED)
        return o1_rounds(S, R, out, lt, PackedCols{I.M8, I.MB, reinterpret_cast<const uint64_t *>(I.COL)}, I.FC, I.DS,
                         I.stride, dead, true, S.states[lane], resolve);
    else
        return o1_rounds(S, R, out, lt, ByteCols{I.M8, I.MB, dense_col_stride(nd)}, I.FC, I.DS, I.stride, dead, true, S.states[lane], resolve);
}

// The two one-warp order-1 decoders: the small class (packed columns:
// o1s_stream up to kShflMaxNd symbols, o1w_stream<2, packed> up to
// kSmallMaxNd) and the wide class (byte columns, o1w_stream<TPL>). Row
// arrays: 3 nd + 2 rows per buffer; the small class keeps them in static
// shared memory, the wide class right below its word ring in dynamic shared
// memory, sized for the stream's own |D| (the launch reserves them for the
// largest |D| among its streams), so a full-range stream's CTA is ~1.5 KB
// smaller than with rows for |D| = kDenseMax.
template <bool kWide>
__global__ void __launch_bounds__(32)
    dec_o1w_kernel(const uint8_t *__restrict__ src, DecStream *__restrict__ streams,
                   const uint32_t *__restrict__ list, int nlist, const uint8_t *__restrict__ tbl,
                   uint8_t *__restrict__ dst, int *__restrict__ queue, uint32_t ring_off,
                   uint32_t first_polls, uint8_t *__restrict__ mirror) {
    constexpr int kRows = kWide ? 1 : 3 * kSmallMaxNd + 2;
    extern __shared__ __align__(128) uint8_t sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ __align__(16) uint4 s_rows[2][kRows];
    const int lane = threadIdx.x;
    const uint32_t lt = lanemask_lt();
    TableStager st;
    st.init(&bar);
    bool stuck = false;
    for (;;) {
        const int j = pop_job(queue);
        if (j >= nlist) return;
        DecStream &S = streams[list[j]];
        if (stuck) {
            mark_timeout(S);
            continue;
        }
        st.issue(sm, tbl + S.tbl_off, S.tbl_bytes);
        WordRing R;
        R.init(src + S.words_off, S.words_len, sm + ring_off);
        if (!st.wait(first_polls)) {
            stuck = !st.drain();
            mark_timeout(S);
            continue;
        }
        uint8_t *out = dst + S.dst_off;
        int status;
        if constexpr (kWide) {
            const int tpl = (S.nd + kWideLanes - 1) / kWideLanes;
            uint4 *r0 = reinterpret_cast<uint4 *>(sm + ring_off - wide_rows_bytes(S.nd));
            uint4 *r1 = r0 + (3 * S.nd + 2);
            status = tpl <= 2   ? o1w_stream<2, false>(S, sm, R, r0, r1, out, lt)
                     : tpl == 3 ? o1w_stream<3, false>(S, sm, R, r0, r1, out, lt)
                     : tpl == 4 ? o1w_stream<4, false>(S, sm, R, r0, r1, out, lt)
                                : o1w_stream<5, false>(S, sm, R, r0, r1, out, lt);
        } else {
            status = S.nd <= 7            ? o1s_stream<true>(S, sm, R, out, lt)
                     : S.nd <= kShflMaxNd ? o1s_stream<false>(S, sm, R, out, lt)
                                          : o1w_stream<2, true>(S, sm, R, s_rows[0], s_rows[1], out, lt);
        }
        if (lane == 0) S.status = status;
        __syncwarp();
        if (mirror && status == FQXV_RANS_OK) mirror_out(out, mirror + S.dst_off, S.n, lane, 32);
    }
}
static_assert((kDenseMax + kWideLanes - 1) / kWideLanes <= 5, "o1w_stream instantiations cover TPL <= 5");
static_assert((kSmallMaxNd + kWideLanes - 1) / kWideLanes <= 2, "the small class runs o1w_stream<2>");
static_assert(3 * kShflMaxNd + 1 <= 31, "shuffle-resolved chains fit in a warp");

// ---------------------------------------------------------------------------
// order-1, large alphabets: tables stay in global memory (L2), one dependent
// lookup per position.
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(32)
    dec_o1g_kernel(const uint8_t *__restrict__ src, DecStream *__restrict__ streams,
                   const uint32_t *__restrict__ list, int nlist, const uint8_t *__restrict__ tbl,
                   uint8_t *__restrict__ dst, int *__restrict__ queue, uint8_t *__restrict__ mirror) {
    extern __shared__ __align__(128) uint8_t sm[];
    const int lane = threadIdx.x;
    const uint32_t lt = lanemask_lt();
    for (;;) {
        const int j = pop_job(queue);
        if (j >= nlist) return;
        DecStream &S = streams[list[j]];
        const uint8_t *base = tbl + S.tbl_off + kDecO1Base;
        WordRing R;
        R.init(src + S.words_off, S.words_len, sm);
        const uint64_t n = S.n;
        const uint64_t navail = S.words_len / 2;
        const bool all_present = S.nctx == 256;
        uint32_t x = S.states[lane];
        uint8_t *out = dst + S.dst_off;
        uint64_t wp = 0;
        uint32_t t = (uint32_t)S.ctx0;
        int status = FQXV_RANS_OK;
        const uint64_t rounds = (n + 31) / 32;
        for (uint64_t r = 0; r < rounds; r++) {
            R.advance(wp);
            const uint64_t i = r * 32 + lane;
            const bool active = i < n;
            const uint64_t left = n - r * 32;
            const int jmax = left < 32 ? (int)left : 32;
            const uint32_t slot = x & (kTotFreq - 1);
            uint32_t my_t = 0, my_e = 0;
            int absent_at = 32;
#pragma unroll
            for (int k = 0; k < 32; k++) {
                const uint32_t sl = __shfl_sync(0xffffffffu, slot, k);
                if (k < jmax) {
                    if (!all_present && t == 0xffu) {
                        absent_at = k;
                        break;
                    }
                    const uint32_t e16 = __ldg(reinterpret_cast<const uint16_t *>(base + kDecO1Ctx * t) + sl);
                    if (lane == k) {
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
                const uint32_t fc =
                    __ldg(reinterpret_cast<const uint32_t *>(base + kDecO1Ctx * my_t + kDecO1Slot) + sym);
                v = (fc >> kScaleBits) * (x >> kScaleBits) + slot - (fc & (kTotFreq - 1));
            }
            const bool need = valid && v < kRansL;
            if (!renorm_round(v, need, R, wp, navail, lt)) {
                status = FQXV_RANS_E_TRUNCATED;
                break;
            }
            if (absent_at < jmax) {
                status = FQXV_RANS_E_ABSENT_CONTEXT;
                break;
            }
            if (active) {
                out[i] = (uint8_t)(my_e >> 8);
                x = v;
            }
        }
        if (lane == 0) S.status = status;
        __syncwarp();
        if (mirror && status == FQXV_RANS_OK) mirror_out(out, mirror + S.dst_off, S.n, lane, 32);
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

uint32_t dec_smem_bytes(int cls, uint32_t tbl_bytes, int nd) {
    switch (cls) {
        case kClsO0: return 16384 + kRingBytes;
        case kClsO1Dense: return (uint32_t)align_up(tbl_bytes, 128) + kO1Warps * kRingBytes;
        case kClsO1Global: return kRingBytes;
        case kClsO1Small: return (uint32_t)align_up(tbl_bytes, 128) + kRingBytes;
        case kClsO1Wide: return (uint32_t)align_up(tbl_bytes, 128) + wide_rows_bytes(nd) + kRingBytes;
        default: return 0;
    }
}

// Dynamic shared memory of one CTA that leaves no room on its SM for any
// other: the per-block opt-in maximum less the kernel's static shared memory.
// With per_sm > 1: the share that lets exactly per_sm such CTAs fill an SM
// (each CTA also costs its static shared memory and the 1 KB the driver
// reserves per block).
static uint32_t exclusive_bytes(const void *fn, int per_sm) {
    int dev = 0, optin = 0, per_smem = 0;
    cudaFuncAttributes a;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&per_smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        cudaFuncGetAttributes(&a, fn) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int64_t b = (int64_t)optin - (int64_t)a.sharedSizeBytes;
    if (per_sm > 1) b = std::min<int64_t>(b, (int64_t)per_smem / per_sm - 1024 - (int64_t)a.sharedSizeBytes);
    return b > 0 ? (uint32_t)b / 128 * 128 : 0u;
}

uint32_t dec_exclusive_smem(int cls, int per_sm) {
    if (cls == kClsO1Dense) return exclusive_bytes(reinterpret_cast<const void *>(dec_o1d_kernel), per_sm);
    if (cls == kClsO1Small) return exclusive_bytes(reinterpret_cast<const void *>(dec_o1w_kernel<false>), per_sm);
    return 0;
}

// Each decode kernel's dynamic shared-memory limit is raised once per
// device to the largest size any launch uses. Setting it per launch would
// race between host threads that launch the same kernel with different sizes
// (a launch can find the limit lowered by another thread and fail).
static std::mutex g_attr_mu;
static bool g_attr_done[256];

static void ensure_dec_attrs() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) {
        cudaGetLastError();
        return;
    }
    std::lock_guard<std::mutex> lk(g_attr_mu);
    if (g_attr_done[dev]) return;
    cudaFuncSetAttribute(dec_o0_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)dec_smem_bytes(kClsO0, 0));
    cudaFuncSetAttribute(dec_o1d_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)std::max(dec_smem_bytes(kClsO1Dense, kDenseImageMax), dec_exclusive_smem(kClsO1Dense)));
    cudaFuncSetAttribute(dec_o1g_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)dec_smem_bytes(kClsO1Global, 0));
    cudaFuncSetAttribute(dec_o1w_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)std::max(dec_smem_bytes(kClsO1Small, kDenseImageMax), dec_exclusive_smem(kClsO1Small)));
    cudaFuncSetAttribute(dec_o1w_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)dec_smem_bytes(kClsO1Wide, kDenseImageMax));
    // Kernels whose tables live in shared memory take the largest shared-
    // memory share of the SM's L1, so as many streams as fit run per SM (the
    // global-table decoder keeps its L1 for the tables it reads through it).
    cudaFuncSetAttribute(dec_o0_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    cudaFuncSetAttribute(dec_o1d_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    cudaFuncSetAttribute(dec_o1w_kernel<false>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
    cudaFuncSetAttribute(dec_o1w_kernel<true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
    cudaGetLastError();
    g_attr_done[dev] = true;
}

int dec_blocks_per_sm(int cls, uint32_t smem_bytes) {
    ensure_dec_attrs();
    int n = 0;
    cudaError_t e = cudaSuccess;
    switch (cls) {
        case kClsO0:
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dec_o0_kernel, 32, smem_bytes);
            break;
        case kClsO1Dense:
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dec_o1d_kernel, kO1Threads, smem_bytes);
            break;
        case kClsO1Global:
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dec_o1g_kernel, 32, smem_bytes);
            break;
        case kClsO1Small:
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dec_o1w_kernel<false>, 32, smem_bytes);
            break;
        case kClsO1Wide:
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dec_o1w_kernel<true>, 32, smem_bytes);
            break;
        default:
            break;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return n > 0 ? n : 1;
}

void launch_dec_parse(const uint8_t *src, DecStream *streams, int nstreams, uint8_t *tbl, int grid,
                      cudaStream_t s) {
    if (nstreams <= 0) return;
    dec_parse_kernel<<<grid, kParseThreads, 0, s>>>(src, streams, nstreams, tbl);
}

void launch_dec_run(int cls, const uint8_t *src, DecStream *streams, const uint32_t *list, int nlist,
                    const uint8_t *tbl, uint8_t *dst, int *queue, int grid, uint32_t smem_bytes,
                    uint32_t first_polls, uint8_t *mirror, cudaStream_t s) {
    if (nlist <= 0 || grid <= 0) return;
    ensure_dec_attrs();
    switch (cls) {
        case kClsO0:
            dec_o0_kernel<<<grid, 32, smem_bytes, s>>>(src, streams, list, nlist, tbl, dst, queue, first_polls,
                                                       mirror);
            break;
        case kClsO1Dense:
            dec_o1d_kernel<<<grid, kO1Threads, smem_bytes, s>>>(src, streams, list, nlist, tbl, dst, queue,
                                                                smem_bytes - kO1Warps * kRingBytes, first_polls,
                                                                mirror);
            break;
        case kClsO1Global:
            dec_o1g_kernel<<<grid, 32, smem_bytes, s>>>(src, streams, list, nlist, tbl, dst, queue, mirror);
            break;
        case kClsO1Small:
            dec_o1w_kernel<false><<<grid, 32, smem_bytes, s>>>(src, streams, list, nlist, tbl, dst, queue,
                                                                smem_bytes - kRingBytes, first_polls, mirror);
            break;
        case kClsO1Wide:
            dec_o1w_kernel<true><<<grid, 32, smem_bytes, s>>>(src, streams, list, nlist, tbl, dst, queue,
                                                               smem_bytes - kRingBytes, first_polls, mirror);
            break;
        default:
            break;
    }
}

}  // namespace fqxv
