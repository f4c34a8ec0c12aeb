// Encode path of the B200 rANS Nx16 coder.
//
// Stages (each one launch over the whole batch):
//   1. enc_model_kernel   one CTA per block: order-0 histogram (warp-private
//      shared-memory atomics with run-length folding), exact normalisation,
//      encode tables; for order-1 a dense |U| x |U| pair histogram and one
//      normalised model per present context.
//   2. enc_run_kernel     one warp per (block, order) job taken from a device
//      work queue (jobs sorted largest first): lane l owns state l and walks
//      the rounds from the last to the first, emitting renorm words with a
//      ballot/popc compaction written back to front into a word scratch.
//   3. enc_select_scan    encoded sizes, order selection, exclusive scan.
//   4. enc_pack_kernel    one CTA per block: header, frequency tables, states
//      and words written to their compacted place in the output arena.
// Byte format and arithmetic follow crates/fqxv-rans/src/scalar.rs:29-140 and
// model.rs:52-264.
#include <cooperative_groups.h>
#include <mutex>

#include "rans_common.cuh"
#include "rans_internal.cuh"

namespace fqxv {

namespace {

__device__ __forceinline__ void unpack16(const uint4 v, uint32_t b[16]) {
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int k = 0; k < 16; k++) b[k] = (w[k >> 2] >> (8 * (k & 3))) & 0xffu;
}

// Visit positions [lo, hi) of the block p in 16-byte aligned vector chunks
// (one per thread per step) and in single bytes for the unaligned head and
// the tail. For every byte the visitor gets (previous byte or 0 at position
// 0, byte); runs of equal keys are folded into one shared-memory atomic.
template <class KeyFn, class AddFn, class EmitFn, class Emit16Fn>
__device__ __forceinline__ void histogram_pass(const uint8_t *__restrict__ p, uint64_t lo, uint64_t hi, KeyFn key,
                                               AddFn add, EmitFn emit, Emit16Fn emit16) {
    if (hi <= lo) return;
    const uint64_t n = hi - lo;
    const uint64_t mis = (uint64_t)(uintptr_t)(p + lo) & 15u;
    uint64_t head = mis ? 16 - mis : 0;
    if (head > n) head = n;
    const uint64_t body = (n - head) / 16;
    const uint64_t tail0 = lo + head + body * 16;
    for (uint64_t i = lo + threadIdx.x; i < lo + head; i += blockDim.x) {
        const uint32_t k = key(i ? p[i - 1] : 0u, p[i]);
        emit(i, k);
        add(k, 1u);
    }
    for (uint64_t i = tail0 + threadIdx.x; i < hi; i += blockDim.x) {
        const uint32_t k = key(i ? p[i - 1] : 0u, p[i]);
        emit(i, k);
        add(k, 1u);
    }
    for (uint64_t c = threadIdx.x; c < body; c += blockDim.x) {
        const uint64_t pos = lo + head + 16 * c;
        const uint4 v = __ldg(reinterpret_cast<const uint4 *>(p + pos));
        uint32_t b[16];
        unpack16(v, b);
        uint32_t prev = pos ? (uint32_t)p[pos - 1] : 0u;
        uint32_t ks[16];
        uint32_t k0 = key(prev, b[0]);
        ks[0] = k0;
        uint32_t run = 1;
#pragma unroll
        for (int k = 1; k < 16; k++) {
            const uint32_t kk = key(b[k - 1], b[k]);
            ks[k] = kk;
            if (kk != k0) {
                add(k0, run);
                k0 = kk;
                run = 1;
            } else {
                run++;
            }
        }
        add(k0, run);
        emit16(pos, ks);
    }
}

__device__ __forceinline__ uint2 enc_entry(uint32_t f, uint32_t cum) {
    // avx2.rs:245-264: magic = floor((2^32 - 1) / f); fc = (f << 12) | cum.
    // Absent symbols get an all-zero entry (their cum can be 4096, which
    // would otherwise spill into the frequency field).
    if (f == 0) return make_uint2(0u, 0u);
    return make_uint2(0xffffffffu / f, (f << kScaleBits) | cum);
}

}  // namespace

// Model of one block per thread-block cluster of kModelCluster CTAs: every
// CTA histograms its slice of the block into its own shared memory and the
// slices are summed through distributed shared memory. Counts: scalar.rs:30-33
// (order-0) and :62-80 (order-1); normalisation: model.rs:213-264.
__global__ void __launch_bounds__(kModelThreads)
    enc_model_kernel(const uint8_t *__restrict__ src, EncBlock *__restrict__ blocks,
                     const uint32_t *__restrict__ order, int nblocks, uint8_t *__restrict__ tbl,
                     uint32_t *__restrict__ hist_scratch, uint16_t *__restrict__ keys) {
    namespace cg = cooperative_groups;
    constexpr int W = kModelThreads / 32;
    constexpr int kSmemU = 64;
    __shared__ uint32_t h0[W][256];
    __shared__ uint32_t h1[kSmemU * kSmemU];
    __shared__ uint32_t part[256];      // this CTA's order-0 counts
    __shared__ uint32_t cnt[256];       // the block's order-0 counts
    __shared__ uint32_t rowbuf[W][kSmemU];
    __shared__ uint8_t umap[256];
    __shared__ int s_nu, s_nctx;
    cg::cluster_group cl = cg::this_cluster();
    const int C = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int cid = blockIdx.x / C, ncl = gridDim.x / C;
    uint32_t *gh = hist_scratch + (size_t)cid * 65536;

    for (int bi = cid; bi < nblocks; bi += ncl) {
        const int b = order[bi];
        const uint8_t *p = src + blocks[b].src_off;
        const uint64_t n = blocks[b].n;
        const int mode = blocks[b].mode;
        uint8_t *T = tbl + blocks[b].tbl_off;
        const uint64_t lo = n * (uint64_t)rank / C, hi = n * (uint64_t)(rank + 1) / C;

        for (int i = tid; i < W * 256; i += blockDim.x) (&h0[0][0])[i] = 0;
        if (tid == 0) s_nctx = 0;
        __syncthreads();
        uint32_t *hw = h0[warp];
        histogram_pass(
            p, lo, hi, [](uint32_t, uint32_t c) { return c; },
            [&](uint32_t k, uint32_t r) { atomicAdd(&hw[k], r); }, [](uint64_t, uint32_t) {},
            [](uint64_t, const uint32_t *) {});
        __syncthreads();
        if (tid < 256) {
            uint32_t t = 0;
#pragma unroll
            for (int w = 0; w < W; w++) t += h0[w][tid];
            part[tid] = t;
        }
        cl.sync();  // every slice's counts are in place
        if (tid < 256) {
            uint32_t t = 0;
            for (int r = 0; r < C; r++) t += cl.map_shared_rank(part, r)[tid];
            cnt[tid] = t;
        }
        __syncthreads();

        if (mode != FQXV_RANS_ORDER1 && rank == 0 && warp == 0) {
            uint32_t f[8], cum[8];
            bool present;
            warp_normalize(cnt, 256, f, cum, present);
            uint2 *T0 = reinterpret_cast<uint2 *>(T + kTblO0);
#pragma unroll
            for (int k = 0; k < 8; k++) T0[lane * 8 + k] = enc_entry(f[k], cum[k]);
        }
        if (mode == FQXV_RANS_ORDER0) {
            cl.sync();  // no CTA rewrites `part` while another still reads it
            continue;
        }

        // Order-1 (scalar.rs:62-80). U = occurring bytes plus context 0, in
        // ascending byte order; contexts and symbols share that dense index.
        // Every CTA derives the same map from the same counts.
        if (warp == 0) {
            uint32_t flags = 0;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int s = lane * 8 + k;
                if (cnt[s] != 0 || s == 0) flags |= 1u << k;
            }
            const uint32_t c = __popc(flags);
            uint32_t base = warp_incl_scan(c) - c;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int s = lane * 8 + k;
                umap[s] = (flags >> k) & 1u ? (uint8_t)(base++) : (uint8_t)0xff;
            }
            if (lane == 31) s_nu = (int)(base);
        }
        __syncthreads();
        const int nu = s_nu;
        auto pair = [&](uint32_t prev, uint32_t c) { return (uint32_t)umap[prev] * nu + umap[c]; };
        // the order-1 table index of every position, for the encode (when
        // the caller gave scratch for it); indexed from src rounded down to
        // 16 bytes, so a 16-byte input chunk's indices are one aligned 32 B
        uint16_t *kb = keys ? keys + ((uintptr_t)src & 15u) + blocks[b].src_off : nullptr;
        auto emit = [&](uint64_t i, uint32_t k) {
            if (kb) kb[i] = (uint16_t)k;
        };
        auto emit16 = [&](uint64_t pos, const uint32_t *k) {
            if (!kb) return;
            uint4 *d = reinterpret_cast<uint4 *>(kb + pos);
            d[0] = make_uint4(k[0] | k[1] << 16, k[2] | k[3] << 16, k[4] | k[5] << 16, k[6] | k[7] << 16);
            d[1] = make_uint4(k[8] | k[9] << 16, k[10] | k[11] << 16, k[12] | k[13] << 16, k[14] | k[15] << 16);
        };
        uint2 *T1 = reinterpret_cast<uint2 *>(T + kTblO1);
        if (rank == 0 && tid < 256) T[kTblUmap + tid] = umap[tid];
        if (nu <= kSmemU) {
            // pair counts of this slice in shared memory, rows summed over
            // the cluster; context rows are spread over all warps of it
            for (int i = tid; i < nu * nu; i += blockDim.x) h1[i] = 0;
            __syncthreads();
            histogram_pass(p, lo, hi, pair, [&](uint32_t k, uint32_t r) { atomicAdd(&h1[k], r); }, emit, emit16);
            cl.sync();
            for (int t = warp + W * rank; t < nu; t += W * C) {
                for (int u = lane; u < nu; u += 32) {
                    uint32_t v = 0;
                    for (int r = 0; r < C; r++) v += cl.map_shared_rank(h1, r)[t * nu + u];
                    rowbuf[warp][u] = v;
                }
                __syncwarp();
                uint32_t f[8], cum[8];
                bool present;
                warp_normalize(rowbuf[warp], nu, f, cum, present);
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int u = lane * 8 + k;
                    if (u < nu) T1[(size_t)t * nu + u] = enc_entry(f[k], cum[k]);
                }
                if (lane == 0 && present) atomicAdd(&s_nctx, 1);
                __syncwarp();
            }
        } else if (rank == 0) {
            // large alphabets: the cluster's first CTA counts the whole block
            // in global scratch
            for (int i = tid; i < nu * nu; i += blockDim.x) gh[i] = 0;
            __syncthreads();
            histogram_pass(p, 0, n, pair, [&](uint32_t k, uint32_t r) { atomicAdd(&gh[k], r); }, emit, emit16);
            __syncthreads();
            for (int t = warp; t < nu; t += W) {
                uint32_t f[8], cum[8];
                bool present;
                warp_normalize(gh + (size_t)t * nu, nu, f, cum, present);
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int u = lane * 8 + k;
                    if (u < nu) T1[(size_t)t * nu + u] = enc_entry(f[k], cum[k]);
                }
                if (lane == 0 && present) atomicAdd(&s_nctx, 1);
            }
        }
        cl.sync();  // all rows done; s_nctx final in every CTA
        if (rank == 0 && tid == 0) {
            int k = 0;
            for (int r = 0; r < C; r++) k += *cl.map_shared_rank(&s_nctx, r);
            blocks[b].nu = nu;
            blocks[b].nctx = k;
        }
        cl.sync();  // no CTA rewrites shared state while another still reads it
    }
}

// One encode step of a lane (scalar.rs:120-127 with the map of
// model.rs:125-133, computed as avx2.rs:383-393): a state at or above
// x_max = f << 20 gives up its low 16 bits (at most one word), then
// x' = v + cum + q (4096 - f) with q = v / f from the magic reciprocal and one
// correction. Both quotient candidates (with and without the renorm shift)
// start at once, so the chain is compare -> select -> multiply -> compare ->
// select. Returns whether the lane emits a word (its pre-step low 16 bits).
__device__ __forceinline__ bool enc_step(uint32_t &x, uint2 e, bool active) {
    const uint32_t f = e.y >> kScaleBits;
    const uint32_t cum = e.y & (kTotFreq - 1);
    const uint32_t xmax_m1 = (f << 20) - 1u;  // wraps to 2^32 - 1 for f == 4096: never emits
    const uint32_t cmpl = kTotFreq - f;
    const bool need = active && x > xmax_m1;
    const uint32_t xs = x >> 16;
    const uint32_t qa = __umulhi(x, e.x);
    const uint32_t qb = __umulhi(xs, e.x);
    const uint32_t v = need ? xs : x;
    const uint32_t q0 = need ? qb : qa;
    const uint32_t r0 = v - q0 * f;
    const uint32_t x0 = v + cum + q0 * cmpl;
    const uint32_t xn = r0 >= f ? x0 + cmpl : x0;
    if (active) x = xn;
    return need;
}

// Emit the words of one round: the reference emits them high lane first
// (scalar.rs:39-43), so stored below `wptr` they land in ascending lane order
// and the finished region is already in decode order (scalar.rs:134-139).
__device__ __forceinline__ void enc_emit(bool need, uint32_t word, uint16_t *__restrict__ &wptr, uint32_t lt) {
    const uint32_t mask = __ballot_sync(0xffffffffu, need);
    wptr -= __popc(mask);
    st_u16_if(need, wptr + __popc(mask & lt), word);
}

// Reverse-order encode of one block by one warp (scalar.rs:39-43 / :84-90).
// Lane l owns state l; round r covers positions [32r, 32r + 32). The partial
// top round goes first, then the full rounds from the last to the first in
// chunks of 16 whose symbols are loaded one chunk ahead. Word emission (a
// warp vote per round) is kept off the state chain: a chunk records its
// emit flags and pre-step states, and its words are written while the next
// chunk's states are computed.
template <int ORDER, bool SMEM_TAB, bool KEYS>
__device__ __forceinline__ void encode_warp(const uint8_t *__restrict__ p, uint64_t n,
                                            const uint2 *__restrict__ tab,
                                            const uint8_t *__restrict__ umap, uint32_t nu,
                                            const uint16_t *__restrict__ keys,
                                            uint16_t *__restrict__ words, uint64_t word_end,
                                            uint64_t &nwords, uint32_t &state) {
    const int lane = threadIdx.x & 31;
    const uint32_t lt = lanemask_lt();
    uint32_t x = kRansL;
    uint16_t *wptr = words + word_end;
    const int64_t full = (int64_t)(n / 32);
    const uint32_t rem = (uint32_t)(n % 32);
    // Table entry of symbol s with predecessor `prev` (order-1: scalar.rs:85).
    // With KEYS, `s` is already the position's order-1 table index.
    auto entry = [&](uint32_t s, uint32_t prev) -> uint2 {
        if (ORDER == 0) return tab[s];
        const uint32_t idx = KEYS ? s : (uint32_t)umap[prev] * nu + umap[s];
        return SMEM_TAB ? tab[idx] : __ldg(tab + idx);
    };
    // symbol (or table index) of position i, and its context byte
    auto sym_at = [&](uint64_t i) -> uint32_t { return KEYS ? (uint32_t)keys[i] : (uint32_t)__ldg(p + i); };
    constexpr bool CTX = ORDER == 1 && !KEYS;
    if (rem) {
        const uint64_t i = (uint64_t)full * 32 + lane;
        const bool active = lane < (int)rem;
        const uint32_t s = active ? sym_at(i) : 0u;
        uint32_t prev = 0;
        if (CTX) prev = (active && i > 0) ? (uint32_t)__ldg(p + i - 1) : 0u;
        const uint2 e = active ? entry(s, prev) : make_uint2(0u, 0u);
        const uint32_t x_before = x;
        const bool need = enc_step(x, e, active);
        enc_emit(need, x_before, wptr, lt);
    }
    // cur/nxt: symbols of this chunk and the next; for order-1 also the
    // byte before each position (its context, scalar.rs:85; 0 before the
    // first byte), loaded with them instead of exchanged between lanes.
    uint32_t cur[16], nxt[16], curp[16], nxtp[16], wv[16], pwv[16];
    uint32_t pbits = 0;  // emit flags of the previous chunk (bit k = round rt + 16 - k)
#pragma unroll
    for (int k = 0; k < 16; k++) {
        const int64_t r = full - 1 - k;
        const uint64_t i = (uint64_t)r * 32 + lane;
        cur[k] = r >= 0 ? sym_at(i) : 0u;
        curp[k] = (CTX && r >= 0 && i > 0) ? (uint32_t)__ldg(p + i - 1) : 0u;
        pwv[k] = 0;
    }
    for (int64_t rt = full - 1; rt >= 0; rt -= 16) {
        if (rt >= 32) {
            const uint64_t ic = (uint64_t)(rt - 16) * 32 + lane;
#pragma unroll
            for (int k = 0; k < 16; k++) {
                nxt[k] = sym_at(ic - 32 * k);
                if (CTX) nxtp[k] = (uint32_t)__ldg(p + ic - 32 * k - 1);
            }
        } else {
#pragma unroll
            for (int k = 0; k < 16; k++) {
                const int64_t r = rt - 16 - k;
                const uint64_t i = (uint64_t)r * 32 + lane;
                nxt[k] = r >= 0 ? sym_at(i) : 0u;
                nxtp[k] = (CTX && r >= 0 && i > 0) ? (uint32_t)__ldg(p + i - 1) : 0u;
            }
        }
        const bool whole = rt >= 15;
        // The chunk's table entries first: they depend only on the symbols,
        // so their loads overlap one another instead of stalling the state
        // chain one round at a time (a warp issues in order).
        uint2 ent[16];
#pragma unroll
        for (int k = 0; k < 16; k++) ent[k] = entry(cur[k], CTX ? curp[k] : 0u);
        uint32_t bits = 0;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            wv[k] = x;
            const bool active = whole || k <= rt;
            if (enc_step(x, ent[k], active)) bits |= 1u << k;
            enc_emit((pbits >> k) & 1u, pwv[k], wptr, lt);
        }
        pbits = bits;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            cur[k] = nxt[k];
            curp[k] = nxtp[k];
            pwv[k] = wv[k];
        }
    }
#pragma unroll
    for (int k = 0; k < 16; k++) enc_emit((pbits >> k) & 1u, pwv[k], wptr, lt);
    nwords = (uint64_t)((words + word_end) - wptr);
    state = x;
}

// Order-1 reverse encode without a per-position key array (scalar.rs:84-90):
// the context of position i is byte i - 1, which for lanes 1-31 is the
// symbol the lane below holds in the same round, and for lane 0 the symbol
// lane 31 holds one round lower -- one shuffle per round instead of a second
// byte load. A chunk's table entries (dense index of the context and the
// symbol, then the table) are computed while the chunk above it runs its
// state chain, from symbols loaded one chunk earlier (the byte below a
// chunk's lowest round too), so neither the loads nor the lookups stand
// between one chunk's chain and the next.
template <bool SMEM_TAB>
__device__ __forceinline__ void encode_warp_o1(const uint8_t *__restrict__ p, uint64_t n,
                                               const uint2 *__restrict__ tab, const uint8_t *__restrict__ umap,
                                               uint32_t nu, uint16_t *__restrict__ words, uint64_t word_end,
                                               uint64_t &nwords, uint32_t &state) {
    const int lane = threadIdx.x & 31;
    const uint32_t lt = lanemask_lt();
    const uint32_t below = (uint32_t)(lane + 31) & 31u;  // the lane holding the byte before this lane's
    uint32_t x = kRansL;
    uint16_t *wptr = words + word_end;
    const int64_t full = (int64_t)(n / 32);
    const uint32_t rem = (uint32_t)(n % 32);
    auto tabat = [&](uint32_t idx) -> uint2 { return SMEM_TAB ? tab[idx] : __ldg(tab + idx); };
    auto sym = [&](int64_t r) -> uint32_t { return r >= 0 ? (uint32_t)__ldg(p + (uint64_t)r * 32 + lane) : 0u; };
    if (rem) {
        const uint64_t i = (uint64_t)full * 32 + lane;
        const bool active = lane < (int)rem;
        const uint32_t s = active ? (uint32_t)__ldg(p + i) : 0u;
        const uint32_t prev = (active && i > 0) ? (uint32_t)__ldg(p + i - 1) : 0u;
        const uint2 e = active ? tabat((uint32_t)umap[prev] * nu + umap[s]) : make_uint2(0u, 0u);
        const uint32_t x_before = x;
        const bool need = enc_step(x, e, active);
        enc_emit(need, x_before, wptr, lt);
    }
    // entries of the chunk whose top round is rt, from its symbols cs[k]
    // (round rt - k) and the symbol of round rt - 16 (lane 31's is the
    // context of lane 0 in round rt - 15); rounds below 0 hold symbol 0,
    // which is the context of position 0
    auto entries = [&](const uint32_t (&cs)[16], uint32_t low, uint2 (&ent)[16]) {
        uint32_t u[17];
#pragma unroll
        for (int k = 0; k < 16; k++) u[k] = umap[cs[k]];
        u[16] = umap[low];
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const uint32_t up = __shfl_sync(0xffffffffu, lane == 31 ? u[k + 1] : u[k], below);
            ent[k] = tabat(up * nu + u[k]);
        }
    };
    // c1: symbols of the chunk below the running one; lo1: the round below
    // c1's lowest (its lane 31 holds the context of c1's lowest lane 0).
    // Both are loaded one chunk before `entries` reads them.
    uint32_t c1[16], c2[16], wv[16], pwv[16], lo1, lo2;
    uint2 ent[16], entn[16];
    uint32_t pbits = 0;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        c1[k] = sym(full - 1 - k);
        pwv[k] = 0;
    }
    {
        uint32_t c0[16];
#pragma unroll
        for (int k = 0; k < 16; k++) c0[k] = c1[k];
#pragma unroll
        for (int k = 0; k < 16; k++) c1[k] = sym(full - 17 - k);
        lo1 = sym(full - 33);
        entries(c0, c1[0], ent);
    }
    for (int64_t rt = full - 1; rt >= 0; rt -= 16) {
#pragma unroll
        for (int k = 0; k < 16; k++) c2[k] = sym(rt - 32 - k);
        lo2 = sym(rt - 48);
        entries(c1, lo1, entn);
        const bool whole = rt >= 15;
        uint32_t bits = 0;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            wv[k] = x;
            const bool active = whole || k <= rt;
            if (enc_step(x, ent[k], active)) bits |= 1u << k;
            enc_emit((pbits >> k) & 1u, pwv[k], wptr, lt);
        }
        pbits = bits;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            ent[k] = entn[k];
            c1[k] = c2[k];
            pwv[k] = wv[k];
        }
        lo1 = lo2;
    }
#pragma unroll
    for (int k = 0; k < 16; k++) enc_emit((pbits >> k) & 1u, pwv[k], wptr, lt);
    nwords = (uint64_t)((words + word_end) - wptr);
    state = x;
}

// Order-1 tables of alphabets up to kEncO1SmemNu symbols are copied into
// the warp's slice of dynamic shared memory; larger ones are read through L1.
constexpr uint32_t kEncO1SmemNu = 45;
constexpr uint32_t kEncO1TabBytes = (kEncO1SmemNu * kEncO1SmemNu * 8 + 127) / 128 * 128;

__global__ void __launch_bounds__(kEncWarpsPerCta * 32)
    enc_run_kernel(const uint8_t *__restrict__ src, EncBlock *__restrict__ blocks,
                   const EncJob *__restrict__ jobs, int njobs, const uint8_t *__restrict__ tbl,
                   uint16_t *__restrict__ words, int *__restrict__ queue, const uint16_t *__restrict__ keys) {
    extern __shared__ __align__(16) uint8_t dsm[];
    __shared__ uint2 s_tab[kEncWarpsPerCta][256];
    __shared__ uint8_t s_umap[kEncWarpsPerCta][256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (;;) {
        int j = 0;
        if (lane == 0) j = atomicAdd(queue, 1);
        j = __shfl_sync(0xffffffffu, j, 0);
        if (j >= njobs) return;
        const EncJob job = jobs[j];
        EncBlock &B = blocks[job.block];
        const uint64_t n = B.n;
        const uint8_t *p = src + B.src_off;
        const uint8_t *T = tbl + B.tbl_off;
        const uint64_t word_end = B.word_off[job.order] + n;
        uint64_t nw = 0;
        uint32_t st = kRansL;
        if (n) {
            if (job.order == 0) {
                const uint2 *T0 = reinterpret_cast<const uint2 *>(T + kTblO0);
#pragma unroll
                for (int k = 0; k < 8; k++) s_tab[warp][lane * 8 + k] = T0[lane * 8 + k];
                __syncwarp();
                encode_warp<0, true, false>(p, n, s_tab[warp], nullptr, 0, nullptr, words, word_end, nw, st);
            } else {
#pragma unroll
                for (int k = 0; k < 8; k++) s_umap[warp][lane * 8 + k] = T[kTblUmap + lane * 8 + k];
                const uint32_t nu = (uint32_t)B.nu;
                const uint2 *T1 = reinterpret_cast<const uint2 *>(T + kTblO1);
                if (nu <= kEncO1SmemNu) {
                    uint2 *t = reinterpret_cast<uint2 *>(dsm + warp * kEncO1TabBytes);
                    for (uint32_t i = lane; i < nu * nu; i += 32) t[i] = T1[i];
                    __syncwarp();
                    if (keys)
                        encode_warp<1, true, true>(p, n, t, s_umap[warp], nu, keys + ((uintptr_t)src & 15u) + B.src_off, words,
                                                   word_end, nw, st);
                    else
                        encode_warp_o1<true>(p, n, t, s_umap[warp], nu, words, word_end, nw, st);
                } else {
                    __syncwarp();
                    if (keys)
                        encode_warp<1, false, true>(p, n, T1, s_umap[warp], nu, keys + ((uintptr_t)src & 15u) + B.src_off, words,
                                                    word_end, nw, st);
                    else
                        encode_warp_o1<false>(p, n, T1, s_umap[warp], nu, words, word_end, nw, st);
                }
            }
        }
        B.states[job.order][lane] = st;
        if (lane == 0) B.nwords[job.order] = nw;
        __syncwarp();
    }
}

__global__ void __launch_bounds__(1024)
    enc_select_scan_kernel(EncBlock *__restrict__ blocks, int nblocks, uint64_t *__restrict__ total) {
    __shared__ uint64_t wtot[32];
    __shared__ uint64_t carry;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nblocks; base += 1024) {
        const int b = base + tid;
        uint64_t size = 0;
        if (b < nblocks) {
            EncBlock &B = blocks[b];
            const uint64_t n = B.n;
            const uint64_t s0 = n ? kHdr + kO0Tables + kStatesBytes + 2 * B.nwords[0] : kHdr;
            const uint64_t s1 =
                n ? kHdr + kO1Bitmap + kO1Table * (uint64_t)B.nctx + kStatesBytes + 2 * B.nwords[1] : kHdr;
            int ch;
            switch (B.mode) {
                case FQXV_RANS_ORDER0: ch = 0; break;
                case FQXV_RANS_ORDER1: ch = 1; break;
                case FQXV_RANS_BEST_TIE0: ch = s1 < s0 ? 1 : 0; break;
                default: ch = s1 <= s0 ? 1 : 0; break;
            }
            B.out_size[0] = s0;
            B.out_size[1] = s1;
            B.chosen = ch;
            size = ch ? s1 : s0;
        }
        const uint64_t incl = warp_incl_scan_u64(size);
        if (lane == 31) wtot[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const uint64_t v = wtot[lane];
            const uint64_t vi = warp_incl_scan_u64(v);
            wtot[lane] = vi - v;
            if (lane == 31) wtot[31] = vi - v;  // keep exclusive; chunk total below
        }
        __syncthreads();
        const uint64_t excl = carry + wtot[warp] + incl - size;
        if (b < nblocks) blocks[b].out_off = excl;
        __syncthreads();
        if (tid == 1023) carry = excl + size;
        __syncthreads();
    }
    if (tid == 0) *total = carry;
}

// Bytes [lo, hi) of src to the same positions of dst, by the whole CTA:
// 4-byte stores at aligned destination addresses, each assembled from the
// two aligned source words it straddles (a load never leaves the aligned
// word of a byte it needs).
__device__ __forceinline__ void cta_copy(uint8_t *__restrict__ dst, const uint8_t *__restrict__ src, uint64_t lo,
                                         uint64_t hi) {
    const uint32_t tid = threadIdx.x;
    if (hi <= lo) return;
    const uint64_t lead = (4u - ((uintptr_t)(dst + lo) & 3u)) & 3u;
    const uint64_t head = lead < hi - lo ? lead : hi - lo;
    if (tid < head) dst[lo + tid] = src[lo + tid];
    const uint64_t a = lo + head;
    const uint64_t nw = (hi - a) / 4;
    const uint32_t sh = (uint32_t)((uintptr_t)(src + a) & 3u);
    const uint32_t *s4 = reinterpret_cast<const uint32_t *>((uintptr_t)(src + a) & ~(uintptr_t)3);
    uint32_t *d4 = reinterpret_cast<uint32_t *>(dst + a);
    if (sh == 0) {
        for (uint64_t j = tid; j < nw; j += blockDim.x) d4[j] = s4[j];
    } else {
        for (uint64_t j = tid; j < nw; j += blockDim.x) d4[j] = __funnelshift_r(s4[j], s4[j + 1], 8 * sh);
    }
    const uint64_t t = a + 4 * nw;
    if (tid < hi - t) dst[t + tid] = src[t + tid];
}

// One work item per (block, part): part 0 writes the header, tables and
// states, and every part copies its slice of the renorm words.
__global__ void __launch_bounds__(kPackThreads)
    enc_pack_kernel(const EncBlock *__restrict__ blocks, int nblocks, const uint8_t *__restrict__ tbl,
                    const uint16_t *__restrict__ words, uint8_t *__restrict__ dst) {
    __shared__ uint8_t present[256];
    __shared__ uint8_t rowctx[256];
    __shared__ int s_k;
    const int tid = threadIdx.x;
    const int nitems = nblocks * kPackParts;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int b = item / kPackParts, part = item % kPackParts;
        const EncBlock &B = blocks[b];
        const int o = B.chosen;
        const uint64_t n = B.n;
        uint8_t *d = dst + B.out_off;
        if (n == 0 && part != 0) continue;
        const uint64_t hdr = o == 0 ? kHdr + kO0Tables : kHdr + kO1Bitmap + kO1Table * (uint64_t)B.nctx;
        if (part != 0) {
            const uint64_t W2 = 2 * B.nwords[o];
            const uint64_t lo = (W2 * part / kPackParts) & ~(uint64_t)15;
            const uint64_t hi = part + 1 == kPackParts ? W2 : (W2 * (part + 1) / kPackParts) & ~(uint64_t)15;
            const uint8_t *ws = reinterpret_cast<const uint8_t *>(words + B.word_off[o] + n - B.nwords[o]);
            cta_copy(d + hdr + kStatesBytes, ws, lo, hi);
            continue;
        }
        if (tid == 0) d[0] = (uint8_t)o;
        if (tid >= 1 && tid <= 8) d[tid] = (uint8_t)(n >> (8 * (tid - 1)));
        if (n == 0) continue;
        const uint8_t *T = tbl + B.tbl_off;
        uint64_t off = kHdr;
        if (o == 0) {
            const uint2 *T0 = reinterpret_cast<const uint2 *>(T + kTblO0);
            for (int s = tid; s < 256; s += blockDim.x) {
                const uint32_t f = T0[s].y >> kScaleBits;
                d[off + 2 * s] = (uint8_t)f;
                d[off + 2 * s + 1] = (uint8_t)(f >> 8);
            }
            off += kO0Tables;
        } else {
            // scalar.rs:96-107: presence bitmap, then one table per present
            // context in ascending context order.
            const int nu = B.nu;
            const uint8_t *um = T + kTblUmap;
            const uint2 *T1 = reinterpret_cast<const uint2 *>(T + kTblO1);
            // With all 256 byte values in U the map is the identity and 0xFF
            // is a real index, not the "absent" marker.
            const bool full = nu == 256;
            if (tid < 256) {
                const uint32_t u = um[tid];
                bool pr = false;
                if (full || u != 0xffu)
                    for (int v = 0; v < nu && !pr; v++) pr = T1[(size_t)u * nu + v].y != 0;
                present[tid] = pr;
            }
            __syncthreads();
            if (tid < 32) {
                uint32_t bits = 0, cntp = 0;
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    bits |= (uint32_t)present[tid * 8 + k] << k;
                    cntp += present[tid * 8 + k];
                }
                d[off + tid] = (uint8_t)bits;
                uint32_t base = warp_incl_scan(cntp) - cntp;
#pragma unroll
                for (int k = 0; k < 8; k++)
                    if (present[tid * 8 + k]) rowctx[base++] = (uint8_t)(tid * 8 + k);
                if (tid == 31) s_k = (int)base;
            }
            __syncthreads();
            off += kO1Bitmap;
            const int K = s_k;
            for (int e = tid; e < K * 256; e += blockDim.x) {
                const uint32_t u = um[rowctx[e >> 8]];
                const uint32_t us = um[e & 255];
                const uint32_t f = (full || us != 0xffu) ? (T1[(size_t)u * nu + us].y >> kScaleBits) : 0u;
                d[off + 2 * (uint64_t)e] = (uint8_t)f;
                d[off + 2 * (uint64_t)e + 1] = (uint8_t)(f >> 8);
            }
            off += kO1Table * (uint64_t)K;
        }
        if (tid < kStates) {
            const uint32_t x = B.states[o][tid];
#pragma unroll
            for (int k = 0; k < 4; k++) d[off + 4 * tid + k] = (uint8_t)(x >> (8 * k));
        }
        off += kStatesBytes;
        const uint64_t W2 = 2 * B.nwords[o];
        const uint8_t *ws = reinterpret_cast<const uint8_t *>(words + B.word_off[o] + n - B.nwords[o]);
        cta_copy(d + off, ws, 0, kPackParts == 1 ? W2 : (W2 / kPackParts) & ~(uint64_t)15);
        __syncthreads();
    }
}

cudaError_t launch_enc_model(const uint8_t *src, EncBlock *blocks, const uint32_t *order, int nblocks,
                             uint8_t *tbl, uint32_t *hist_scratch, uint16_t *keys, int grid, int cluster,
                             cudaStream_t s) {
    if (nblocks <= 0) return cudaSuccess;
    // `grid` clusters of `cluster` CTAs
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid * (unsigned)cluster, 1, 1);
    cfg.blockDim = dim3(kModelThreads, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, enc_model_kernel, src, blocks, order, nblocks, tbl, hist_scratch, keys);
}

void launch_enc_run(const uint8_t *src, EncBlock *blocks, const EncJob *jobs, int njobs,
                    const uint8_t *tbl, uint16_t *words, int *queue, const uint16_t *keys, int grid,
                    cudaStream_t s) {
    if (njobs <= 0) return;
    static std::mutex mu;
    static bool done[256];
    int dev = 0;
    cudaGetDevice(&dev);
    {
        // raised once per device: a per-launch setting would race between
        // host threads (see the decode launchers)
        std::lock_guard<std::mutex> lk(mu);
        if (dev >= 0 && dev < 256 && !done[dev]) {
            cudaFuncSetAttribute(enc_run_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(kEncWarpsPerCta * kEncO1TabBytes));
            // three CTAs per SM (the register limit) need ~225 KB of shared memory
            cudaFuncSetAttribute(enc_run_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
            cudaGetLastError();
            done[dev] = true;
        }
    }
    enc_run_kernel<<<grid, kEncWarpsPerCta * 32, kEncWarpsPerCta * kEncO1TabBytes, s>>>(src, blocks, jobs, njobs,
                                                                                       tbl, words, queue, keys);
}

void launch_enc_select_scan(EncBlock *blocks, int nblocks, uint64_t *total, cudaStream_t s) {
    enc_select_scan_kernel<<<1, 1024, 0, s>>>(blocks, nblocks, total);
}

void launch_enc_pack(EncBlock *blocks, int nblocks, const uint8_t *tbl, const uint16_t *words,
                     uint8_t *dst, int grid, cudaStream_t s) {
    if (nblocks <= 0) return;
    enc_pack_kernel<<<grid, kPackThreads, 0, s>>>(blocks, nblocks, tbl, words, dst);
}

}  // namespace fqxv
