// The extended stream format on the GPU: a new format tag (first byte
// 0x80 | flags) with no counterpart in the reference, which writes one
// format only (32 states, flag-less [u8 order][u64 n] header:
// crates/fqxv-rans/src/model.rs:19, scalar.rs:8-20). Layout and selection
// rules are those of the CPU definition in oracle/rans_x.c; parity with it is
// the only check there is (parity unpinned against the reference).
//
//   [u8 0x80 | flags][u64 n] body           (n == 0: no body)
//   ORDER1 (0x01) cores use the order-1 model; N4 (0x02) cores use 4 states;
//   STRIPE (0x04) four nested streams of the byte planes i % 4 == j;
//   PACK (0x10) [u8 nsym][symbols], codes of 0/1/2/4 bits packed LSB first;
//   RLE (0x08) [u8 nrun][run symbols][u64 nlit][u64 nrb], runs of run
//   symbols become one literal plus a LEB128 (length - 1);
//   CAT (0x20) cores stored raw; otherwise a core is [u64 len][stream].
//
// Design: the transforms are data-parallel byte passes (CTA per block, CUB
// block scans over tiles for RLE); 32-state cores go through the batched
// coder of rans_capi.cu, so they are byte-identical reference streams; 4-state
// cores reuse the model kernel for their tables and run one thread per core
// for the serial four-state chain (a 4-way stream has 4 independent states,
// an eighth of the parallelism of the 32-way format).
#include <algorithm>
#include <cstring>
#include <vector>

#include <cub/block/block_scan.cuh>

#include "../../include/fqxv_rans_x_gpu.h"
#include "rans_common.cuh"
#include "rans_ctx.cuh"

namespace fqxv {
namespace {

constexpr int kXThreads = 512;
constexpr int kXItems = 4;                   // positions per thread per RLE tile
constexpr int kXTile = kXThreads * kXItems;  // positions per RLE tile

// One array being transformed / coded (a block, a STRIPE plane, or a core).
struct XItem {
    uint64_t src_off;    // input bytes (n of them) in the source arena
    uint64_t n;
    uint64_t work_off;   // work arena: [packed m | literals <= m | run bytes <= m]
    uint64_t m;          // array after PACK (n without PACK)
    uint64_t nlit, nrb;  // RLE arrays
    uint32_t nsym, nrun; // PACK symbols, RLE run symbols
    uint32_t flags;
    int32_t status;
    uint8_t syms[16];
    uint32_t runbits[8];  // RLE run-symbol bitmap
};

__device__ __forceinline__ int pack_bits(uint32_t nsym) { return nsym <= 1 ? 0 : nsym <= 2 ? 1 : nsym <= 4 ? 2 : 4; }
__host__ inline int pack_bits_h(uint32_t nsym) { return nsym <= 1 ? 0 : nsym <= 2 ? 1 : nsym <= 4 ? 2 : 4; }

// Symbols present in each item's input (ascending); more than 16 leaves
// nsym = their count and no symbol list (PACK is not applicable).
__global__ void __launch_bounds__(256) x_symset_kernel(const uint8_t *__restrict__ src, XItem *__restrict__ items,
                                                        int nitems) {
    __shared__ uint32_t seen[8];
    const int tid = threadIdx.x;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        XItem &I = items[it];
        if (tid < 8) seen[tid] = 0;
        __syncthreads();
        const uint8_t *p = src + I.src_off;
        for (uint64_t i = tid; i < I.n; i += blockDim.x) {
            const uint32_t s = p[i];
            if (!((seen[s >> 5] >> (s & 31)) & 1u)) atomicOr(&seen[s >> 5], 1u << (s & 31));
        }
        __syncthreads();
        if (tid == 0) {
            uint32_t k = 0;
            for (int s = 0; s < 256; s++)
                if ((seen[s >> 5] >> (s & 31)) & 1u) {
                    if (k < 16) I.syms[k] = (uint8_t)s;
                    k++;
                }
            I.nsym = k;
        }
        __syncthreads();
    }
}

// PACK: packed byte j of item = codes of positions j * per .. j * per + per - 1.
__global__ void __launch_bounds__(256) x_pack_kernel(const uint8_t *__restrict__ src, uint8_t *__restrict__ work,
                                                      const XItem *__restrict__ items, int nitems) {
    __shared__ uint8_t code[256];
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const XItem &I = items[it];
        if (I.nsym > 16) continue;
        __syncthreads();
        for (int s = threadIdx.x; s < 256; s += blockDim.x) code[s] = 0;
        __syncthreads();
        if (threadIdx.x < I.nsym) code[I.syms[threadIdx.x]] = (uint8_t)threadIdx.x;
        __syncthreads();
        const int bits = pack_bits(I.nsym);
        if (bits == 0) continue;
        const uint32_t per = 8u / (uint32_t)bits;
        const uint8_t *p = src + I.src_off;
        uint8_t *q = work + I.work_off;
        for (uint64_t j = threadIdx.x; j < I.m; j += blockDim.x) {
            uint32_t v = 0;
            for (uint32_t t = 0; t < per; t++) {
                const uint64_t i = j * per + t;
                if (i < I.n) v |= (uint32_t)code[p[i]] << (t * (uint32_t)bits);
            }
            q[j] = (uint8_t)v;
        }
    }
}

// Run symbols of each item's array (after PACK): occurrences above twice the
// number of maximal runs.
__global__ void __launch_bounds__(256) x_runsym_kernel(const uint8_t *__restrict__ src,
                                                        const uint8_t *__restrict__ work, XItem *__restrict__ items,
                                                        int nitems) {
    __shared__ unsigned long long occ[256], runs[256];
    const int tid = threadIdx.x;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        XItem &I = items[it];
        if (I.status) continue;
        const uint8_t *a = (I.flags & FQXV_X_PACK) ? work + I.work_off : src + I.src_off;
        occ[tid] = 0;
        runs[tid] = 0;
        __syncthreads();
        for (uint64_t i = tid; i < I.m; i += blockDim.x) {
            const uint32_t s = a[i];
            atomicAdd(&occ[s], 1ull);
            if (i == 0 || a[i - 1] != s) atomicAdd(&runs[s], 1ull);
        }
        __syncthreads();
        const bool r = occ[tid] > 2 * runs[tid];
        const uint32_t bal = __ballot_sync(0xffffffffu, r);
        if ((tid & 31) == 0) I.runbits[tid >> 5] = bal;
        __syncthreads();
        if (tid == 0) {
            uint32_t k = 0;
            for (int w = 0; w < 8; w++) k += __popc(I.runbits[w]);
            I.nrun = k;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ uint32_t varint_len(uint64_t v) {
    uint32_t k = 1;
    while (v >= 0x80) {
        v >>= 7;
        k++;
    }
    return k;
}

struct RleAgg {
    uint64_t start;   // index of the current run's first position (max-scan)
    uint32_t lits;    // literals emitted
    uint32_t rbytes;  // run bytes emitted
};

struct RleOp {
    __device__ __forceinline__ RleAgg operator()(const RleAgg &a, const RleAgg &b) const {
        return RleAgg{a.start > b.start ? a.start : b.start, a.lits + b.lits, a.rbytes + b.rbytes};
    }
};

// RLE of each item's array in tiles of kXTile positions, one CTA per item:
// a literal at every position of a non-run symbol and at the first position
// of every run of a run symbol; at the last position of such a run its
// length - 1 as a LEB128 varint. One block scan per tile gives each
// position's run start (max) and its literal and run-byte offsets (sums).
__global__ void __launch_bounds__(kXThreads) x_rle_kernel(const uint8_t *__restrict__ src,
                                                           uint8_t *__restrict__ work, XItem *__restrict__ items,
                                                           int nitems) {
    using Scan = cub::BlockScan<RleAgg, kXThreads>;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ uint32_t runbits[8];
    __shared__ uint64_t c_start, c_lits, c_rbytes;  // totals of the tiles before
    const int tid = threadIdx.x;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        XItem &I = items[it];
        if (I.status) continue;
        const uint8_t *a = (I.flags & FQXV_X_PACK) ? work + I.work_off : src + I.src_off;
        uint8_t *lits = work + I.work_off + I.m;
        uint8_t *rb = lits + I.m;
        const uint64_t m = I.m;
        if (tid < 8) runbits[tid] = I.runbits[tid];
        if (tid == 0) c_start = c_lits = c_rbytes = 0;
        __syncthreads();
        for (uint64_t base = 0; base < m; base += kXTile) {
            uint32_t s[kXItems];
            bool st[kXItems], en[kXItems], isr[kXItems];
            RleAgg loc = {0, 0, 0};
            uint64_t lastst = 0;
            for (int k = 0; k < kXItems; k++) {
                const uint64_t i = base + (uint64_t)tid * kXItems + k;
                const bool in = i < m;
                s[k] = in ? a[i] : 0u;
                st[k] = in && (i == 0 || a[i - 1] != s[k]);
                en[k] = in && (i + 1 == m || a[i + 1] != s[k]);
                isr[k] = in && ((runbits[s[k] >> 5] >> (s[k] & 31)) & 1u);
                if (st[k]) lastst = i;
            }
            loc.start = lastst;
            // per-position literal and run-byte counts need the run start,
            // known only after the scan: count them after it
            RleAgg pre;
            RleAgg tot;
            Scan(tmp).ExclusiveScan(loc, pre, RleAgg{0, 0, 0}, RleOp(), tot);
            __syncthreads();
            uint64_t start = pre.start > c_start ? pre.start : c_start;
            uint32_t nl = 0, nb = 0;
            uint64_t lens[kXItems];
            for (int k = 0; k < kXItems; k++) {
                const uint64_t i = base + (uint64_t)tid * kXItems + k;
                if (st[k]) start = i;
                lens[k] = i - start;  // run length - 1 at the run's last position
                if (i < m) {
                    if (!isr[k] || st[k]) nl++;
                    if (isr[k] && en[k]) nb += varint_len(lens[k]);
                }
            }
            RleAgg cnt = {0, nl, nb}, cpre, ctot;
            __syncthreads();
            Scan(tmp).ExclusiveScan(cnt, cpre, RleAgg{0, 0, 0}, RleOp(), ctot);
            uint64_t lo = c_lits + cpre.lits, bo = c_rbytes + cpre.rbytes;
            for (int k = 0; k < kXItems; k++) {
                const uint64_t i = base + (uint64_t)tid * kXItems + k;
                if (i >= m) break;
                if (!isr[k] || st[k]) lits[lo++] = (uint8_t)s[k];
                if (isr[k] && en[k]) {
                    uint64_t v = lens[k];
                    while (v >= 0x80) {
                        rb[bo++] = (uint8_t)(v | 0x80);
                        v >>= 7;
                    }
                    rb[bo++] = (uint8_t)v;
                }
            }
            __syncthreads();
            if (tid == 0) {
                c_start = tot.start > c_start ? tot.start : c_start;
                c_lits += ctot.lits;
                c_rbytes += ctot.rbytes;
            }
            __syncthreads();
        }
        if (tid == 0) {
            I.nlit = c_lits;
            I.nrb = c_rbytes;
        }
        __syncthreads();
    }
}

// Copies [src + off, + n) of each item to dst + dst_off (one CTA per item).
struct XCopy {
    uint64_t src_off, dst_off, n;
};
__global__ void __launch_bounds__(256) x_copy_kernel(const uint8_t *__restrict__ src, uint8_t *__restrict__ dst,
                                                      const XCopy *__restrict__ c, int n) {
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        const uint8_t *s = src + c[k].src_off;
        uint8_t *d = dst + c[k].dst_off;
        for (uint64_t i = threadIdx.x; i < c[k].n; i += blockDim.x) d[i] = s[i];
    }
}

// STRIPE: plane j of item (bytes i % 4 == j) to plane_off[4 * it + j].
__global__ void __launch_bounds__(256) x_stripe_kernel(const uint8_t *__restrict__ src, uint8_t *__restrict__ dst,
                                                        const uint64_t *__restrict__ in_off,
                                                        const uint64_t *__restrict__ in_n,
                                                        const uint64_t *__restrict__ plane_off, int nitems) {
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const uint8_t *p = src + in_off[it];
        const uint64_t n = in_n[it];
        for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) dst[plane_off[4 * it + (i & 3)] + (i >> 2)] = p[i];
    }
}

__global__ void __launch_bounds__(256) x_unstripe_kernel(const uint8_t *__restrict__ planes,
                                                          uint8_t *__restrict__ dst,
                                                          const uint64_t *__restrict__ out_off,
                                                          const uint64_t *__restrict__ out_n,
                                                          const uint64_t *__restrict__ plane_off, int nitems) {
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        uint8_t *d = dst + out_off[it];
        const uint64_t n = out_n[it];
        for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) d[i] = planes[plane_off[4 * it + (i & 3)] + (i >> 2)];
    }
}

// ---- 4-state cores ---------------------------------------------------------

// One warp per core, lanes 0-3 holding states 0-3: the reverse encode of
// scalar.rs:29-111 with 4 states (state i % 4 codes position i), tables from
// the model kernel. A round is positions 4r .. 4r + 3, coded from the top
// round down; the CPU definition emits position 4r + 3's word first, so
// stored below the write pointer the round's words land in ascending lane
// order, handed out by a vote. The next round's table entries are loaded
// before this round's state updates. Words end below word_off + n, in
// decode order.
__global__ void __launch_bounds__(128) x_n4_run_kernel(const uint8_t *__restrict__ src, EncBlock *__restrict__ blocks,
                                                        int nblocks, const uint8_t *__restrict__ tbl,
                                                        uint16_t *__restrict__ words) {
    const int lane = threadIdx.x & 31;
    const int b = blockIdx.x * 4 + (int)(threadIdx.x >> 5);
    if (b >= nblocks) return;
    EncBlock &B = blocks[b];
    const uint64_t n = B.n;
    const int o = B.mode == FQXV_RANS_ORDER1 ? 1 : 0;
    const uint8_t *p = src + B.src_off;
    const uint8_t *T = tbl + B.tbl_off;
    const uint2 *T0 = reinterpret_cast<const uint2 *>(T + kTblO0);
    const uint2 *T1 = reinterpret_cast<const uint2 *>(T + kTblO1);
    const uint8_t *um = T + kTblUmap;
    const uint32_t nu = (uint32_t)B.nu;
    const uint32_t lt = (1u << lane) - 1u;
    auto entry = [&](uint64_t i) -> uint2 {
        const uint32_t sy = p[i];
        if (o == 0) return T0[sy];
        const uint32_t c = i ? p[i - 1] : 0u;
        return T1[(size_t)um[c] * nu + um[sy]];
    };
    uint32_t x = kRansL;
    uint16_t *const end = words + B.word_off[o] + n;
    uint16_t *w = end;
    // one position of lane's state: emits the pre-step low 16 bits when the
    // state would pass x_max = f << 20 (never for f = 4096)
    auto step = [&](uint2 e, bool active) {
        const uint32_t f = e.y >> kScaleBits, cum = e.y & (kTotFreq - 1);
        uint32_t v = x;
        const bool need = active && (uint64_t)v >= ((uint64_t)f << 20);
        const uint32_t mask = __ballot_sync(0xffffffffu, need);
        w -= __popc(mask);
        if (need) {
            w[__popc(mask & lt)] = (uint16_t)v;
            v >>= 16;
        }
        if (active) {
            uint32_t q = __umulhi(v, e.x);
            uint32_t r = v - q * f;
            if (r >= f) {
                q++;
                r -= f;
            }
            x = (q << kScaleBits) + r + cum;
        }
    };
    const uint64_t full = n / 4;
    const uint32_t rem = (uint32_t)(n % 4);
    if (rem) {
        const bool active = lane < (int)rem;
        step(active ? entry(4 * full + lane) : make_uint2(0u, 0u), active);
    }
    const bool mine = lane < 4;
    uint2 e = (full && mine) ? entry(4 * (full - 1) + lane) : make_uint2(0u, 0u);
    for (uint64_t r = full; r-- > 0;) {
        const uint2 en = (r && mine) ? entry(4 * (r - 1) + lane) : make_uint2(0u, 0u);
        step(e, mine);
        e = en;
    }
    if (mine) B.states[o][lane] = x;
    if (lane == 0) {
        B.nwords[o] = (uint64_t)(end - w);
        B.chosen = o;
    }
}

// Writes one 4-state core per block: [2 | order][u64 n][tables][4 states][words].
__global__ void __launch_bounds__(256) x_n4_pack_kernel(const EncBlock *__restrict__ blocks, int nblocks,
                                                         const uint8_t *__restrict__ tbl,
                                                         const uint16_t *__restrict__ words,
                                                         uint8_t *__restrict__ dst,
                                                         const uint64_t *__restrict__ out_off) {
    __shared__ uint8_t present[256];
    __shared__ uint8_t rowctx[256];
    __shared__ int s_k;
    const int tid = threadIdx.x;
    for (int b = blockIdx.x; b < nblocks; b += gridDim.x) {
        const EncBlock &B = blocks[b];
        const int o = B.chosen;
        const uint64_t n = B.n;
        uint8_t *d = dst + out_off[b];
        if (tid == 0) d[0] = (uint8_t)(2 | o);
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
            const int nu = B.nu;
            const uint8_t *um = T + kTblUmap;
            const uint2 *T1 = reinterpret_cast<const uint2 *>(T + kTblO1);
            const bool full = nu == 256;
            {
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
        if (tid < 16) d[off + tid] = (uint8_t)(B.states[o][tid >> 2] >> (8 * (tid & 3)));
        off += 16;
        const uint16_t *ws = words + B.word_off[o] + n - B.nwords[o];
        for (uint64_t k = tid; k < B.nwords[o]; k += blockDim.x) {
            d[off + 2 * k] = (uint8_t)ws[k];
            d[off + 2 * k + 1] = (uint8_t)(ws[k] >> 8);
        }
        __syncthreads();
    }
}

// Decode side of a 4-state core. One CTA per core: its tables checked in the
// reference's order (model.rs:160-174, scalar.rs:180-198) and expanded into
// slot -> symbol rows (in shared memory when the launch reserved room for
// the core's tables, else in global scratch), then the chain of
// scalar.rs:200-238 with 4 states. Statuses as the CPU definition.
struct XN4Dec {
    uint64_t src_off, len;    // the core stream
    uint64_t dst_off, cap;    // its output
    uint64_t scratch_off;     // rows: K x (4096 B slot map + 256 x u32 freq << 12 | cum)
    uint64_t n;
    int32_t status;
    int32_t pad;
};
constexpr uint64_t kN4Row = 4096 + 1024;
constexpr uint64_t kN4SmemRows = 32;

__global__ void __launch_bounds__(256) x_n4_decode_kernel(const uint8_t *__restrict__ src, XN4Dec *__restrict__ cores,
                                                           int ncores, uint8_t *__restrict__ scratch,
                                                           uint8_t *__restrict__ dst, int ksm) {
    extern __shared__ __align__(16) uint8_t xsm[];  // ksm rows: cores of at most ksm tables keep them here
    __shared__ uint16_t ctxidx[256];
    __shared__ int s_k;
    __shared__ uint32_t wsum[8];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int ci = blockIdx.x; ci < ncores; ci += gridDim.x) {
        XN4Dec &C = cores[ci];
        const uint8_t *p = src + C.src_off;
        const uint64_t L = C.len;
        int status = FQXV_RANS_OK;
        if (L < 9) status = FQXV_RANS_E_TRUNCATED;
        const int order = L >= 9 ? (p[0] & 1) : 0;
        const uint64_t n = L >= 9 ? ld_u64_le(p + 1) : 0;
        if (status != FQXV_RANS_OK || n == 0) {
            if (tid == 0) {
                C.status = status;
                C.n = 0;
            }
            __syncthreads();
            continue;
        }
        uint64_t pos = kHdr;
        if (tid == 0) s_k = 1;
        __syncthreads();
        if (order) {
            if (L < pos + kO1Bitmap) {
                status = FQXV_RANS_E_TRUNCATED;
            } else if (tid == 0) {
                int k = 0;
                for (int c = 0; c < 256; c++) ctxidx[c] = ((p[pos + c / 8] >> (c % 8)) & 1) ? (uint16_t)k++ : 0xffff;
                s_k = k;
            }
            pos += kO1Bitmap;
        } else if (tid < 256) {
            ctxidx[tid] = 0;
        }
        __syncthreads();
        const int K = s_k;
        uint8_t *rows = K <= ksm ? xsm : scratch + C.scratch_off;
        // one table at a time by the whole CTA: the first failing table
        // decides the status, as the sequential reads do
        for (int t = 0; t < K && status == FQXV_RANS_OK; t++) {
            if (L < pos + kO1Table) {
                status = FQXV_RANS_E_TRUNCATED;
                break;
            }
            const uint8_t *q = p + pos;
            const uint32_t f = (uint32_t)q[2 * tid] | ((uint32_t)q[2 * tid + 1] << 8);
            const uint32_t incl = warp_incl_scan(f);
            if (lane == 31) wsum[warp] = incl;
            __syncthreads();
            uint32_t base = 0, tot = 0;
            for (int w = 0; w < 8; w++) {
                if (w < warp) base += wsum[w];
                tot += wsum[w];
            }
            const uint32_t cum = base + incl - f;
            status = tot > kTotFreq ? FQXV_RANS_E_FREQ_EXCEEDS : tot != kTotFreq ? FQXV_RANS_E_FREQ_SUM : FQXV_RANS_OK;
            if (status == FQXV_RANS_OK) {
                uint8_t *row = rows + (uint64_t)t * kN4Row;
                uint32_t *fc = reinterpret_cast<uint32_t *>(row + 4096);
                fc[tid] = (f << kScaleBits) | cum;
                for (uint32_t k = 0; k < f; k++) row[cum + k] = (uint8_t)tid;
            }
            pos += kO1Table;
            __syncthreads();
        }
        if (status == FQXV_RANS_OK && L < pos + 16) status = FQXV_RANS_E_TRUNCATED;
        if (status == FQXV_RANS_OK && n > C.cap) status = FQXV_RANS_E_ALLOC;
        __syncthreads();
        // Order-0 cores: lanes 0-3 of warp 0 hold the four states and decode
        // a round of four positions at once; the round's renorm words are
        // handed out in lane order by a vote (one word at most per state:
        // once every state is at least 2^16, v = f (x >> 12) + slot - cum is
        // at least 16, so one 16-bit word lifts it past 2^16 again). Rounds
        // run this way while a whole round and its four words fit; thread 0
        // finishes the rest, and order-1 cores (a chain of contexts), one
        // position at a time with every check of the CPU definition.
        uint32_t xl = 0;
        uint64_t i0 = 0;
        if (warp == 0 && status == FQXV_RANS_OK) {
            if (lane < 4) xl = ld_u32_le(p + pos + 4 * lane);
            const bool fast = order == 0 && __all_sync(0xffffffffu, lane >= 4 || xl >= kRansL);
            if (fast) {
                const uint8_t *row = rows;
                const uint32_t *fcr = reinterpret_cast<const uint32_t *>(rows + 4096);
                uint8_t *out = dst + C.dst_off;
                const uint32_t lt = (1u << lane) - 1u;
                uint64_t wp = pos + 16;
                while (i0 + 4 <= n && wp + 8 <= L) {
                    uint32_t sy = 0, v = 0;
                    bool need = false;
                    if (lane < 4) {
                        const uint32_t slot = xl & (kTotFreq - 1);
                        sy = row[slot];
                        const uint32_t fc = fcr[sy];
                        v = (fc >> kScaleBits) * (xl >> kScaleBits) + slot - (fc & (kTotFreq - 1));
                        need = v < kRansL;
                    }
                    const uint32_t mask = __ballot_sync(0xffffffffu, need);
                    if (need) {
                        const uint64_t at = wp + 2 * __popc(mask & lt);
                        v = (v << 16) | (uint32_t)p[at] | ((uint32_t)p[at + 1] << 8);
                    }
                    if (lane < 4) {
                        out[i0 + lane] = (uint8_t)sy;
                        xl = v;
                    }
                    wp += 2 * (uint64_t)__popc(mask);
                    i0 += 4;
                }
                pos = wp - 16;  // the serial part below skips the states again
            }
        }
        uint32_t xs4[4];
        for (int k = 0; k < 4; k++) xs4[k] = __shfl_sync(0xffffffffu, xl, k);
        if (tid == 0) {
            if (status == FQXV_RANS_OK) {
                uint32_t x[4];
                for (int k = 0; k < 4; k++) x[k] = xs4[k];
                pos += 16;
                uint8_t *out = dst + C.dst_off;
                uint32_t ctx = 0;
                for (uint64_t i = i0; i < n; i++) {
                    const uint32_t t = ctxidx[ctx];
                    if (t == 0xffffu) {
                        status = FQXV_RANS_E_ABSENT_CONTEXT;
                        break;
                    }
                    const uint8_t *row = rows + (uint64_t)t * kN4Row;
                    const uint32_t xs = x[i & 3];
                    const uint32_t slot = xs & (kTotFreq - 1);
                    const uint32_t s = row[slot];
                    const uint32_t fc = reinterpret_cast<const uint32_t *>(row + 4096)[s];
                    uint32_t v = (fc >> kScaleBits) * (xs >> kScaleBits) + slot - (fc & (kTotFreq - 1));
                    while (v < kRansL) {
                        if (L < pos + 2) {
                            status = FQXV_RANS_E_TRUNCATED;
                            break;
                        }
                        v = (v << 16) | ((uint32_t)p[pos] | ((uint32_t)p[pos + 1] << 8));
                        pos += 2;
                    }
                    if (status) break;
                    x[i & 3] = v;
                    out[i] = (uint8_t)s;
                    ctx = s;
                }
            }
            C.status = status;
            C.n = status == FQXV_RANS_OK ? n : 0;
        }
        __syncthreads();
    }
}

// The 4-state decoder's shared-memory limit, raised once per device.
void ensure_n4_attr() {
    static std::mutex mu;
    static bool done[256];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) {
        cudaGetLastError();
        return;
    }
    std::lock_guard<std::mutex> lk(mu);
    if (done[dev]) return;
    cudaFuncSetAttribute(x_n4_decode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(kN4SmemRows * kN4Row));
    cudaGetLastError();
    done[dev] = true;
}

// Inverse RLE: literals + run bytes -> the array. One CTA per item, tiles of
// literals: a block scan gives each literal's output offset (its run length)
// and its varint's offset in the run bytes (one varint per run-symbol
// literal, located by counting the terminating bytes of the run-byte array
// in a first pass).
struct XUnrle {
    uint64_t lit_off, nlit, rb_off, nrb, out_off, m;
    uint32_t runbits[8];
    int32_t status;
    int32_t pad;
};

__global__ void __launch_bounds__(kXThreads) x_unrle_kernel(uint8_t *__restrict__ work, XUnrle *__restrict__ jobs,
                                                             int njobs, uint64_t *__restrict__ vstart) {
    using Scan = cub::BlockScan<unsigned long long, kXThreads>;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ unsigned long long carry, carry_v;
    __shared__ int s_bad;
    const int tid = threadIdx.x;
    for (int j = blockIdx.x; j < njobs; j += gridDim.x) {
        XUnrle &J = jobs[j];
        const uint8_t *lits = work + J.lit_off;
        const uint8_t *rb = work + J.rb_off;
        uint8_t *out = work + J.out_off;
        uint64_t *vs = vstart + J.rb_off;  // start offset of every varint, by index
        if (tid == 0) {
            carry = 0;
            s_bad = 0;
        }
        __syncthreads();
        // pass 1: varint k starts after the k-th terminating byte
        for (uint64_t base = 0; base < J.nrb; base += kXThreads) {
            const uint64_t i = base + tid;
            const unsigned long long term = i < J.nrb && !(rb[i] & 0x80) ? 1ull : 0ull;
            unsigned long long pre, tot;
            Scan(tmp).ExclusiveSum(term, pre, tot);
            if (i < J.nrb && (i == 0 || !(rb[i - 1] & 0x80))) vs[carry + pre] = i;
            __syncthreads();
            if (tid == 0) carry += tot;
            __syncthreads();
        }
        const uint64_t nvar = carry;
        if (J.nrb && (rb[J.nrb - 1] & 0x80)) s_bad = 1;  // a varint runs past the end
        __syncthreads();
        if (tid == 0) {
            carry = 0;
            carry_v = 0;
        }
        __syncthreads();
        // pass 2: every literal's run length and output offset
        for (uint64_t base = 0; base < J.nlit; base += kXThreads) {
            const uint64_t i = base + tid;
            const bool in = i < J.nlit;
            const uint32_t s = in ? lits[i] : 0u;
            const bool isr = in && ((J.runbits[s >> 5] >> (s & 31)) & 1u);
            unsigned long long vpre, vtot;
            Scan(tmp).ExclusiveSum(isr ? 1ull : 0ull, vpre, vtot);
            __syncthreads();
            uint64_t run = in ? 1 : 0;
            if (isr) {
                const uint64_t k = carry_v + vpre;
                if (k >= nvar) {
                    s_bad = 1;
                } else {
                    uint64_t v = 0;
                    uint32_t sh = 0;
                    for (uint64_t q = vs[k]; q < J.nrb; q++) {
                        if (sh > 56) {
                            s_bad = 1;
                            break;
                        }
                        v |= (uint64_t)(rb[q] & 0x7f) << sh;
                        sh += 7;
                        if (!(rb[q] & 0x80)) break;
                    }
                    run = v + 1;
                    if (run > J.m) s_bad = 1;
                }
            }
            unsigned long long opre, otot;
            Scan(tmp).ExclusiveSum((unsigned long long)run, opre, otot);
            const uint64_t o = carry + opre;
            if (in && !s_bad && o + run <= J.m)
                for (uint64_t q = 0; q < run; q++) out[o + q] = (uint8_t)s;
            __syncthreads();
            if (tid == 0) {
                carry += otot;
                carry_v += vtot;
                if (carry > J.m) s_bad = 1;
            }
            __syncthreads();
        }
        if (tid == 0) J.status = (s_bad || carry != J.m || carry_v != nvar) ? FQXV_RANS_E_X_MALFORMED : 0;
        __syncthreads();
    }
}

// Inverse PACK: output byte i = symbol of code (i % per) of packed byte i / per.
struct XUnpack {
    uint64_t a_off, out_off, n;
    uint32_t nsym;
    int32_t status;
    uint8_t syms[16];
};

__global__ void __launch_bounds__(256) x_unpack_kernel(const uint8_t *__restrict__ work, uint8_t *__restrict__ dst,
                                                        XUnpack *__restrict__ jobs, int njobs) {
    __shared__ int s_bad;
    for (int j = blockIdx.x; j < njobs; j += gridDim.x) {
        XUnpack &J = jobs[j];
        if (threadIdx.x == 0) s_bad = 0;
        __syncthreads();
        const int bits = pack_bits(J.nsym);
        const uint8_t *a = work + J.a_off;
        uint8_t *d = dst + J.out_off;
        bool bad = false;
        for (uint64_t i = threadIdx.x; i < J.n; i += blockDim.x) {
            uint32_t c = 0;
            if (bits) {
                const uint32_t per = 8u / (uint32_t)bits;
                c = (a[i / per] >> ((uint32_t)(i % per) * (uint32_t)bits)) & ((1u << bits) - 1u);
            }
            if (c >= J.nsym) bad = true;
            else d[i] = J.syms[c];
        }
        if (bad) s_bad = 1;
        __syncthreads();
        if (threadIdx.x == 0) J.status = s_bad ? FQXV_RANS_E_X_MALFORMED : 0;
        __syncthreads();
    }
}

// First `H` bytes of every span (fewer for shorter spans) into one buffer.
constexpr uint64_t kHead = 640;
__global__ void __launch_bounds__(128) x_head_kernel(const uint8_t *__restrict__ src, const uint64_t *__restrict__ off,
                                                      const uint64_t *__restrict__ len, int n,
                                                      uint8_t *__restrict__ out) {
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        const uint64_t l = len[k] < kHead ? len[k] : kHead;
        for (uint64_t i = threadIdx.x; i < l; i += blockDim.x) out[(uint64_t)k * kHead + i] = src[off[k] + i];
    }
}


// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

struct Span {
    uint64_t off, len;
};

constexpr uint64_t kNone = ~0ull;

inline void put64(std::vector<uint8_t> &b, uint64_t v) {
    for (int i = 0; i < 8; i++) b.push_back((uint8_t)(v >> (8 * i)));
}
inline uint64_t get64(const uint8_t *p) {
    uint64_t v = 0;
    for (int i = 7; i >= 0; i--) v = (v << 8) | p[i];
    return v;
}

// Device arenas of one extended-format call (grow-only, per context).
struct XBufs {
    DevBuf items, work, core, lit, copies, out, best, planes, misc, vstart, heads;
    HostBuf hbuf;
};

// One batch of copies from `src` to `dst` (device arenas).
int run_copies(fqxv_rans_ctx *ctx, XBufs &B, const uint8_t *src, uint8_t *dst, const std::vector<XCopy> &cps) {
    if (cps.empty()) return FQXV_RANS_OK;
    cudaStream_t s = ctx->stream;
    CK(B.copies.ensure(cps.size() * sizeof(XCopy), s));
    CK(cudaStreamSynchronize(s));
    CK(cudaMemcpyAsync(B.copies.p, cps.data(), cps.size() * sizeof(XCopy), cudaMemcpyHostToDevice, s));
    {
        cudaEvent_t xt_ = ctx->timer.begin(s);
        x_copy_kernel<<<(int)std::min<size_t>(cps.size(), (size_t)ctx->sms * 8), 256, 0, s>>>(
            src, dst, B.copies.as<XCopy>(), (int)cps.size());
        ctx->timer.end(kStXEncode, xt_, s);
    }
    CK(cudaGetLastError());
    return FQXV_RANS_OK;
}

// Bytes from the host into a device arena at `dst_off` positions:
// `lit` holds them back to back, segs gives (lit offset, dst offset, n).
int upload_literals(fqxv_rans_ctx *ctx, XBufs &B, const std::vector<uint8_t> &lit, uint8_t *dst,
                    const std::vector<XCopy> &segs) {
    if (segs.empty()) return FQXV_RANS_OK;
    cudaStream_t s = ctx->stream;
    CK(B.lit.ensure(std::max<size_t>(lit.size(), 16), s));
    CK(cudaStreamSynchronize(s));
    CK(cudaMemcpyAsync(B.lit.p, lit.data(), lit.size(), cudaMemcpyHostToDevice, s));
    return run_copies(ctx, B, B.lit.as<uint8_t>(), dst, segs);
}

// 4-state cores of the arrays `arrs` (spans of d_arena), written back to
// back into `out` (spans returned in `cores`).
int n4_encode(fqxv_rans_ctx *ctx, XBufs &B, const uint8_t *d_arena, const std::vector<Span> &arrs, int order,
              DevBuf &out, std::vector<Span> &cores) {
    cudaStream_t s = ctx->stream;
    const size_t na = arrs.size();
    cores.assign(na, Span{0, 0});
    if (!na) return FQXV_RANS_OK;
    std::vector<EncBlock> hb(na);
    std::vector<uint32_t> ord(na);
    std::vector<uint64_t> ooff(na);
    uint64_t woff = 0, toff = 0, boff = 0;
    for (size_t i = 0; i < na; i++) {
        EncBlock &E = hb[i];
        std::memset(&E, 0, sizeof E);
        E.src_off = arrs[i].off;
        E.n = arrs[i].len;
        E.mode = order;
        E.word_off[0] = E.word_off[1] = woff;
        woff += E.n;
        E.tbl_off = toff;
        toff += align_up(order ? enc_table_bytes(E.n) : kTblUmap, 256);
        ord[i] = (uint32_t)i;
        ooff[i] = boff;
        boff += E.n ? kHdr + (order ? kO1Bitmap + 256 * kO1Table : kO0Tables) + 16 + 2 * E.n : kHdr;
    }
    CK(ctx->e_blocks.ensure(na * sizeof(EncBlock), s));
    CK(ctx->e_order.ensure(na * 4, s));
    CK(ctx->e_tbl.ensure(std::max<uint64_t>(toff, 256), s));
    CK(ctx->e_words.ensure(std::max<uint64_t>(2 * woff, 16), s));
    const int grid = (int)std::min<size_t>(na, (size_t)ctx->sms * 2);
    CK(ctx->e_hist.ensure(order ? (size_t)grid * 65536 * 4 : 256, s));
    CK(B.misc.ensure(na * 8 + 16, s));
    CK(out.ensure(std::max<uint64_t>(boff, 16), s));
    CK(cudaStreamSynchronize(s));
    CK(cudaMemcpyAsync(ctx->e_blocks.p, hb.data(), na * sizeof(EncBlock), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->e_order.p, ord.data(), na * 4, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(B.misc.p, ooff.data(), na * 8, cudaMemcpyHostToDevice, s));
    EncBlock *dB = ctx->e_blocks.as<EncBlock>();
    cudaEvent_t mt_ = ctx->timer.begin(s);
    CK(launch_enc_model(d_arena, dB, ctx->e_order.as<uint32_t>(), (int)na, ctx->e_tbl.as<uint8_t>(),
                        ctx->e_hist.as<uint32_t>(), nullptr, grid, 1, s));
    ctx->timer.end(kStEncModel, mt_, s);
    {
        cudaEvent_t xt_ = ctx->timer.begin(s);
        x_n4_run_kernel<<<(int)((na + 3) / 4), 128, 0, s>>>(d_arena, dB, (int)na, ctx->e_tbl.as<uint8_t>(),
                                                                 ctx->e_words.as<uint16_t>());
        ctx->timer.end(kStXEncode, xt_, s);
    }
    {
        cudaEvent_t xt_ = ctx->timer.begin(s);
        x_n4_pack_kernel<<<grid, 256, 0, s>>>(dB, (int)na, ctx->e_tbl.as<uint8_t>(), ctx->e_words.as<uint16_t>(),
                                               out.as<uint8_t>(), B.misc.as<uint64_t>());
        ctx->timer.end(kStXEncode, xt_, s);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(hb.data(), dB, na * sizeof(EncBlock), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (size_t i = 0; i < na; i++) {
        const EncBlock &E = hb[i];
        uint64_t len = kHdr;
        if (E.n) {
            len += order ? kO1Bitmap + kO1Table * (uint64_t)E.nctx : kO0Tables;
            len += 16 + 2 * E.nwords[order];
        }
        cores[i] = Span{ooff[i], len};
    }
    return FQXV_RANS_OK;
}

// 32-state cores (reference streams) of `arrs`, through the batched coder.
int n32_encode(fqxv_rans_ctx *ctx, const uint8_t *d_arena, const std::vector<Span> &arrs, int order, DevBuf &out,
               std::vector<Span> &cores) {
    cudaStream_t s = ctx->stream;
    const size_t na = arrs.size();
    cores.assign(na, Span{0, 0});
    if (!na) return FQXV_RANS_OK;
    std::vector<fqxv_rans_span> sp(na), os(na);
    for (size_t i = 0; i < na; i++) sp[i] = fqxv_rans_span{arrs[i].off, arrs[i].len};
    const uint64_t bound = fqxv_rans_encode_batch_bound(sp.data(), na, order);
    CK(out.ensure(std::max<uint64_t>(bound, 16), s));
    const int st = encode_batch_locked(ctx, d_arena, sp.data(), na, order, out.as<uint8_t>(), bound, os.data(), nullptr);
    if (st) return st;
    for (size_t i = 0; i < na; i++) cores[i] = Span{os[i].offset, os[i].length};
    return FQXV_RANS_OK;
}

// Streams of `items` (spans of d_src) with flags F (no STRIPE): written back
// to back into `out`; len[i] = kNone where PACK does not apply (more than
// 16 symbols).
int encode_flat(fqxv_rans_ctx *ctx, XBufs &B, const uint8_t *d_src, const std::vector<Span> &items, int F,
                DevBuf &out, std::vector<Span> &res) {
    cudaStream_t s = ctx->stream;
    const size_t ni = items.size();
    res.assign(ni, Span{0, kNone});
    if (!ni) return FQXV_RANS_OK;
    const bool pack = F & FQXV_X_PACK, rle = F & FQXV_X_RLE, cat = F & FQXV_X_CAT;
    std::vector<XItem> hx(ni);
    uint64_t woff = 0;
    for (size_t i = 0; i < ni; i++) {
        XItem &X = hx[i];
        std::memset(&X, 0, sizeof X);
        X.src_off = items[i].off;
        X.n = items[i].len;
        X.m = X.n;
        X.flags = (uint32_t)F;
        X.work_off = woff;
        if (pack || rle) woff += align_up(3 * X.n + 16, 16);
    }
    CK(B.items.ensure(ni * sizeof(XItem), s));
    CK(B.work.ensure(std::max<uint64_t>(woff, 16), s));
    CK(cudaStreamSynchronize(s));
    CK(cudaMemcpyAsync(B.items.p, hx.data(), ni * sizeof(XItem), cudaMemcpyHostToDevice, s));
    XItem *dX = B.items.as<XItem>();
    uint8_t *dW = B.work.as<uint8_t>();
    const int grid = (int)std::min<size_t>(ni, (size_t)ctx->sms * 4);
    if (pack) {
        {
            cudaEvent_t xt_ = ctx->timer.begin(s);
            x_symset_kernel<<<grid, 256, 0, s>>>(d_src, dX, (int)ni);
            ctx->timer.end(kStXEncode, xt_, s);
        }
        CK(cudaMemcpyAsync(hx.data(), dX, ni * sizeof(XItem), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        for (size_t i = 0; i < ni; i++) {
            XItem &X = hx[i];
            if (X.nsym > 16) {
                X.status = 1;
                continue;
            }
            X.m = (X.n * (uint64_t)pack_bits_h(X.nsym) + 7) / 8;
        }
        CK(cudaMemcpyAsync(dX, hx.data(), ni * sizeof(XItem), cudaMemcpyHostToDevice, s));
        {
            cudaEvent_t xt_ = ctx->timer.begin(s);
            x_pack_kernel<<<grid, 256, 0, s>>>(d_src, dW, dX, (int)ni);
            ctx->timer.end(kStXEncode, xt_, s);
        }
    }
    if (rle) {
        {
            cudaEvent_t xt_ = ctx->timer.begin(s);
            x_runsym_kernel<<<grid, 256, 0, s>>>(d_src, dW, dX, (int)ni);
            ctx->timer.end(kStXEncode, xt_, s);
        }
        {
            cudaEvent_t xt_ = ctx->timer.begin(s);
            x_rle_kernel<<<grid, kXThreads, 0, s>>>(d_src, dW, dX, (int)ni);
            ctx->timer.end(kStXEncode, xt_, s);
        }
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(hx.data(), dX, ni * sizeof(XItem), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    // arrays to code: the plain input, the packed bytes, or literals + run bytes
    const uint8_t *arena = (pack || rle) ? dW : d_src;
    std::vector<Span> arrs;
    std::vector<size_t> first(ni, 0);
    for (size_t i = 0; i < ni; i++) {
        const XItem &X = hx[i];
        first[i] = arrs.size();
        if (X.status || X.n == 0) continue;
        if (rle) {
            arrs.push_back(Span{X.work_off + X.m, X.nlit});
            arrs.push_back(Span{X.work_off + 2 * X.m, X.nrb});
        } else {
            arrs.push_back(pack ? Span{X.work_off, X.m} : Span{X.src_off, X.n});
        }
    }
    std::vector<Span> cores;
    DevBuf &cb = B.core;
    if (!cat) {
        const int order = F & FQXV_X_ORDER1 ? 1 : 0;
        const int st = (F & FQXV_X_N4) ? n4_encode(ctx, B, arena, arrs, order, cb, cores)
                                       : n32_encode(ctx, arena, arrs, order, cb, cores);
        if (st) return st;
    }
    // assemble: header and metadata from the host, cores (or raw arrays) copied
    std::vector<uint8_t> lit;
    std::vector<XCopy> lsegs, ccopies;
    uint64_t o = 0;
    for (size_t i = 0; i < ni; i++) {
        const XItem &X = hx[i];
        if (X.status) continue;
        const uint64_t at = o;
        const size_t l0 = lit.size();
        lit.push_back((uint8_t)(0x80 | F));
        put64(lit, X.n);
        if (X.n) {
            if (pack) {
                lit.push_back((uint8_t)X.nsym);
                for (uint32_t k = 0; k < X.nsym; k++) lit.push_back(X.syms[k]);
            }
            if (rle) {
                lit.push_back((uint8_t)X.nrun);
                for (int v = 0; v < 256; v++)
                    if ((X.runbits[v >> 5] >> (v & 31)) & 1u) lit.push_back((uint8_t)v);
                put64(lit, X.nlit);
                put64(lit, X.nrb);
            }
        }
        o += lit.size() - l0;
        const size_t na = X.n == 0 ? 0 : (rle ? 2 : 1);
        for (size_t a = 0; a < na; a++) {
            const Span &A = arrs[first[i] + a];
            if (cat) {
                ccopies.push_back(XCopy{A.off, o, A.len});
                o += A.len;
            } else {
                const Span &C = cores[first[i] + a];
                // the u64 length goes with the literal bytes of this item
                const size_t lb = lit.size();
                put64(lit, C.len);
                lsegs.push_back(XCopy{lb, o, 8});
                o += 8;
                ccopies.push_back(XCopy{C.off, o, C.len});
                o += C.len;
            }
        }
        // header and metadata: the item's first literal bytes (the core
        // lengths follow them in `lit`)
        uint64_t hl = 9;
        if (X.n) {
            if (pack) hl += 1 + X.nsym;
            if (rle) hl += 1 + X.nrun + 16;
        }
        lsegs.push_back(XCopy{l0, at, hl});
        res[i] = Span{at, o - at};
    }
    CK(out.ensure(std::max<uint64_t>(o, 16), s));
    int st = upload_literals(ctx, B, lit, out.as<uint8_t>(), lsegs);
    if (st) return st;
    st = run_copies(ctx, B, cat ? arena : cb.as<uint8_t>(), out.as<uint8_t>(), ccopies);
    if (st) return st;
    CK(cudaStreamSynchronize(s));
    return FQXV_RANS_OK;
}

int encode_best(fqxv_rans_ctx *ctx, XBufs &B, const uint8_t *d_src, const std::vector<Span> &items, bool nested,
                DevBuf &best, std::vector<Span> &res, std::vector<int32_t> &cand);

// STRIPE streams of `items`: planes gathered, each coded by the nested
// selection, then [tag][n][4 x u64 length][4 streams].
int encode_stripe(fqxv_rans_ctx *ctx, XBufs &B, const uint8_t *d_src, const std::vector<Span> &items, int F,
                  DevBuf &out, std::vector<Span> &res) {
    cudaStream_t s = ctx->stream;
    const size_t ni = items.size();
    res.assign(ni, Span{0, kNone});
    std::vector<uint64_t> ioff(ni), in(ni), poff(4 * ni);
    std::vector<Span> planes;
    std::vector<size_t> idx;
    uint64_t po = 0;
    for (size_t i = 0; i < ni; i++) {
        ioff[i] = items[i].off;
        in[i] = items[i].len;
        for (int j = 0; j < 4; j++) {
            const uint64_t nj = (items[i].len + 3 - j) / 4;
            poff[4 * i + j] = po;
            planes.push_back(Span{po, nj});
            po += nj;
        }
        idx.push_back(i);
    }
    XBufs P;  // the nested selection's own arenas
    CK(B.planes.ensure(std::max<uint64_t>(po, 16), s));
    CK(B.misc.ensure((2 * ni + 4 * ni) * 8 + 16, s));
    CK(cudaStreamSynchronize(s));
    uint64_t *dm = B.misc.as<uint64_t>();
    CK(cudaMemcpyAsync(dm, ioff.data(), ni * 8, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dm + ni, in.data(), ni * 8, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dm + 2 * ni, poff.data(), 4 * ni * 8, cudaMemcpyHostToDevice, s));
    {
        cudaEvent_t xt_ = ctx->timer.begin(s);
        x_stripe_kernel<<<(int)std::min<size_t>(ni, (size_t)ctx->sms * 4), 256, 0, s>>>(d_src, B.planes.as<uint8_t>(), dm,
                                                                                         dm + ni, dm + 2 * ni, (int)ni);
        ctx->timer.end(kStXEncode, xt_, s);
    }
    CK(cudaGetLastError());
    DevBuf nb;
    std::vector<Span> nres;
    std::vector<int32_t> ncand;
    int st = encode_best(ctx, P, B.planes.as<uint8_t>(), planes, true, nb, nres, ncand);
    if (st) {
        nb.release();
        return st;
    }
    std::vector<uint8_t> lit;
    std::vector<XCopy> lsegs, copies;
    uint64_t o = 0;
    for (size_t i : idx) {
        const uint64_t at = o;
        const size_t l0 = lit.size();
        lit.push_back((uint8_t)(0x80 | F));  // other flags ride along unused, as written by the definition
        put64(lit, items[i].len);
        if (items[i].len == 0) {  // the header alone, like every empty stream
            lsegs.push_back(XCopy{l0, at, 9});
            o += 9;
            res[i] = Span{at, 9};
            continue;
        }
        for (int j = 0; j < 4; j++) put64(lit, nres[4 * i + j].len);
        lsegs.push_back(XCopy{l0, at, 41});
        o += 41;
        for (int j = 0; j < 4; j++) {
            copies.push_back(XCopy{nres[4 * i + j].off, o, nres[4 * i + j].len});
            o += nres[4 * i + j].len;
        }
        res[i] = Span{at, o - at};
    }
    CK(out.ensure(std::max<uint64_t>(o, 16), s));
    st = upload_literals(ctx, B, lit, out.as<uint8_t>(), lsegs);
    if (!st) st = run_copies(ctx, B, nb.as<uint8_t>(), out.as<uint8_t>(), copies);
    cudaStreamSynchronize(s);
    nb.release();
    for (DevBuf *d : {&P.items, &P.work, &P.core, &P.lit, &P.copies, &P.out, &P.best, &P.planes, &P.misc,
                      &P.vstart, &P.heads})
        d->release();
    P.hbuf.release();
    return st;
}

// The selection of oracle/rans_x.c (candidates 0-9 in order, smallest
// stream, ties to the earlier candidate); `nested` leaves out STRIPE.
int encode_best(fqxv_rans_ctx *ctx, XBufs &B, const uint8_t *d_src, const std::vector<Span> &items, bool nested,
                DevBuf &best, std::vector<Span> &res, std::vector<int32_t> &cand) {
    cudaStream_t s = ctx->stream;
    const size_t ni = items.size();
    res.assign(ni, Span{0, kNone});
    cand.assign(ni, -1);
    if (!ni) return FQXV_RANS_OK;
    // per-item slots in `best` sized for any candidate
    std::vector<uint64_t> slot(ni);
    uint64_t tot = 0;
    for (size_t i = 0; i < ni; i++) {
        slot[i] = tot;
        tot += align_up(fqxv_rans_x_stream_bound(items[i].len), 16);
    }
    CK(best.ensure(std::max<uint64_t>(tot, 16), s));
    std::vector<uint64_t> blen(ni, kNone);
    auto keep = [&](const uint8_t *arena, const std::vector<Span> &r, int c) -> int {
        std::vector<XCopy> cps;
        for (size_t i = 0; i < ni; i++) {
            if (r[i].len == kNone || r[i].len >= blen[i]) continue;
            blen[i] = r[i].len;
            cand[i] = c;
            cps.push_back(XCopy{r[i].off, slot[i], r[i].len});
        }
        const int st = run_copies(ctx, B, arena, best.as<uint8_t>(), cps);
        cudaStreamSynchronize(s);
        return st;
    };
    // candidates 0 and 1: the reference streams, ties to order 0
    {
        std::vector<fqxv_rans_span> sp(ni), os(ni);
        std::vector<int32_t> ord(ni);
        for (size_t i = 0; i < ni; i++) sp[i] = fqxv_rans_span{items[i].off, items[i].len};
        const uint64_t bound = fqxv_rans_encode_batch_bound(sp.data(), ni, FQXV_RANS_BEST_TIE0);
        CK(B.out.ensure(std::max<uint64_t>(bound, 16), s));
        const int st = encode_batch_locked(ctx, d_src, sp.data(), ni, FQXV_RANS_BEST_TIE0, B.out.as<uint8_t>(), bound,
                                           os.data(), ord.data());
        if (st) return st;
        std::vector<Span> r(ni);
        for (size_t i = 0; i < ni; i++) r[i] = Span{os[i].offset, os[i].length};
        std::vector<XCopy> cps;
        for (size_t i = 0; i < ni; i++) {
            blen[i] = r[i].len;
            cand[i] = ord[i];
            cps.push_back(XCopy{r[i].off, slot[i], r[i].len});
        }
        const int st2 = run_copies(ctx, B, B.out.as<uint8_t>(), best.as<uint8_t>(), cps);
        cudaStreamSynchronize(s);
        if (st2) return st2;
    }
    static const int kFlags[10] = {0, 0, FQXV_X_PACK, FQXV_X_PACK | FQXV_X_ORDER1, FQXV_X_RLE,
                                   FQXV_X_RLE | FQXV_X_ORDER1, FQXV_X_PACK | FQXV_X_RLE,
                                   FQXV_X_PACK | FQXV_X_RLE | FQXV_X_ORDER1, FQXV_X_STRIPE, FQXV_X_CAT};
    for (int c = 2; c < 10; c++) {
        if (c == 8 && nested) continue;
        std::vector<Span> r;
        int st;
        if (c == 8) {
            st = encode_stripe(ctx, B, d_src, items, FQXV_X_STRIPE, B.out, r);
            for (size_t i = 0; i < ni; i++)
                if (items[i].len < 4) r[i].len = kNone;  // no STRIPE candidate below 4 bytes
        } else {
            st = encode_flat(ctx, B, d_src, items, kFlags[c], B.out, r);
        }
        if (st) return st;
        st = keep(B.out.as<uint8_t>(), r, c);
        if (st) return st;
    }
    for (size_t i = 0; i < ni; i++) res[i] = Span{slot[i], blen[i]};
    return FQXV_RANS_OK;
}


// ---- decode ----------------------------------------------------------------

// One stream being decoded: a caller's stream, or a STRIPE plane of one.
struct XNode {
    uint64_t src_off, len;   // the stream (a span of the input arena)
    int arena;               // output arena: 0 the caller's, 1 the plane buffer
    uint64_t out_off, cap;
    int parent = -1, plane = 0, level = 0;
    int kind = 0;            // 0 reference stream, 1 flat extended, 2 STRIPE, 3 finished
    int flags = 0;
    uint64_t n = 0;
    int status = 0;
    uint32_t nsym = 0, nrun = 0;
    uint8_t syms[16] = {};
    uint32_t runbits[8] = {};
    uint64_t m = 0, nlit = 0, nrb = 0;
    int ncore = 0;
    uint64_t core_at[2] = {0, 0}, core_len[2] = {0, 0}, arr_len[2] = {0, 0};
    // per core: its header check and its decode, in the order the CPU
    // definition meets them (core 1's header is read only after core 0
    // decoded)
    int cerr[2] = {0, 0}, dstat[2] = {0, 0};
    int post = 0;  // inverse RLE / PACK
    uint64_t arr_off[3] = {0, 0, 0};  // work arena: A (m), literals, run bytes
    int child[4] = {-1, -1, -1, -1};
};

// Reads up to kHead bytes at each (offset, length) of d_src into `out`.
int gather_heads(fqxv_rans_ctx *ctx, XBufs &B, const uint8_t *d_src, const std::vector<Span> &at,
                 std::vector<uint8_t> &out) {
    cudaStream_t s = ctx->stream;
    const size_t k = at.size();
    out.assign(k * kHead, 0);
    if (!k) return FQXV_RANS_OK;
    std::vector<uint64_t> off(k), len(k);
    for (size_t i = 0; i < k; i++) {
        off[i] = at[i].off;
        len[i] = at[i].len;
    }
    CK(B.misc.ensure(2 * k * 8 + 16, s));
    CK(B.heads.ensure(k * kHead, s));
    CK(cudaStreamSynchronize(s));
    uint64_t *dm = B.misc.as<uint64_t>();
    CK(cudaMemcpyAsync(dm, off.data(), k * 8, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dm + k, len.data(), k * 8, cudaMemcpyHostToDevice, s));
    {
        cudaEvent_t xt_ = ctx->timer.begin(s);
        x_head_kernel<<<(int)std::min<size_t>(k, (size_t)ctx->sms * 8), 128, 0, s>>>(d_src, dm, dm + k, (int)k,
                                                                                     B.heads.as<uint8_t>());
        ctx->timer.end(kStXDecode, xt_, s);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out.data(), B.heads.p, k * kHead, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return FQXV_RANS_OK;
}

// Core header checks (oracle/rans_x.c get_core): [u64 len][stream] with the
// declared order and width, and the array's length. `h` holds the bytes at
// `pos` (up to kHead, `avail` of them valid).
int check_core(const uint8_t *h, uint64_t avail, uint64_t L, uint64_t pos, int flags, uint64_t want_n, uint64_t &cl) {
    if (pos > L || L - pos < 8) return FQXV_RANS_E_TRUNCATED;
    cl = get64(h);
    if (cl > L - pos - 8) return FQXV_RANS_E_TRUNCATED;
    if (cl < 9) return FQXV_RANS_E_TRUNCATED;
    if (avail < 17) return FQXV_RANS_E_TRUNCATED;
    const int want = (flags & FQXV_X_N4 ? 2 : 0) | (flags & FQXV_X_ORDER1 ? 1 : 0);
    if (h[8] != want) return FQXV_RANS_E_X_MALFORMED;
    if (get64(h + 9) != want_n) return FQXV_RANS_E_X_MALFORMED;
    return FQXV_RANS_OK;
}

// Parse a node from its first bytes `h` (kHead or its length). STRIPE
// planes become nodes appended to `kids`, numbered from `base`.
void parse_node(XNode &N, const uint8_t *h, std::vector<XNode> &kids, size_t base, int self) {
    const uint64_t L = N.len;
    if (L < 9) {
        N.status = FQXV_RANS_E_TRUNCATED;
        N.kind = 3;
        return;
    }
    if (h[0] < 0x80) {
        N.kind = 0;
        return;
    }
    N.flags = h[0] & 0x7f;
    N.n = get64(h + 1);
    if (N.n == 0) {
        N.kind = 3;
        return;
    }
    if (N.flags & ~FQXV_X_ALL) {
        N.status = FQXV_RANS_E_UNKNOWN_ORDER;
        N.kind = 3;
        return;
    }
    if (N.n > N.cap) {
        N.status = FQXV_RANS_E_ALLOC;
        N.kind = 3;
        return;
    }
    uint64_t pos = 9;
    if (N.flags & FQXV_X_STRIPE) {
        N.kind = 2;
        if (L < pos + 32) {
            N.status = FQXV_RANS_E_TRUNCATED;
            N.kind = 3;
            return;
        }
        uint64_t lens[4];
        for (int j = 0; j < 4; j++) lens[j] = get64(h + pos + 8 * j);
        pos += 32;
        for (int j = 0; j < 4; j++) {
            if (lens[j] > L - pos) {
                // planes before j decode first; their errors come first
                N.child[j] = -2;
                break;
            }
            XNode c;
            c.src_off = N.src_off + pos;
            c.len = lens[j];
            c.arena = 1;
            c.cap = (N.n + 3 - j) / 4;
            c.parent = self;
            c.plane = j;
            c.level = N.level + 1;
            N.child[j] = (int)(base + kids.size());
            kids.push_back(c);
            pos += lens[j];
        }
        return;
    }
    N.kind = 1;
    N.m = N.n;
    if (N.flags & FQXV_X_PACK) {
        if (L < pos + 1) {
            N.status = FQXV_RANS_E_TRUNCATED;
            N.kind = 3;
            return;
        }
        N.nsym = h[pos++];
        if (N.nsym < 1 || N.nsym > 16) {
            N.status = FQXV_RANS_E_X_MALFORMED;
            N.kind = 3;
            return;
        }
        if (L < pos + N.nsym) {
            N.status = FQXV_RANS_E_TRUNCATED;
            N.kind = 3;
            return;
        }
        std::memcpy(N.syms, h + pos, N.nsym);
        pos += N.nsym;
        N.m = (N.n * (uint64_t)pack_bits_h(N.nsym) + 7) / 8;
    }
    if (N.flags & FQXV_X_RLE) {
        if (L < pos + 1) {
            N.status = FQXV_RANS_E_TRUNCATED;
            N.kind = 3;
            return;
        }
        N.nrun = h[pos++];
        if (L < pos + N.nrun + 16) {
            N.status = FQXV_RANS_E_TRUNCATED;
            N.kind = 3;
            return;
        }
        for (uint32_t k = 0; k < N.nrun; k++) N.runbits[h[pos + k] >> 5] |= 1u << (h[pos + k] & 31);
        pos += N.nrun;
        N.nlit = get64(h + pos);
        N.nrb = get64(h + pos + 8);
        pos += 16;
        if (N.nlit > N.m || N.nrb > N.m) {
            N.status = FQXV_RANS_E_X_MALFORMED;
            N.kind = 3;
            return;
        }
        N.ncore = 2;
        N.arr_len[0] = N.nlit;
        N.arr_len[1] = N.nrb;
    } else {
        N.ncore = 1;
        N.arr_len[0] = N.m;
    }
    N.core_at[0] = pos;  // relative to the stream
}

}  // namespace
}  // namespace fqxv

using namespace fqxv;

namespace {

// Per-device arenas of the extended-format calls, kept with the context.
std::mutex g_xmu;

XBufs &xbufs(fqxv_rans_ctx *ctx) {
    std::lock_guard<std::mutex> g(g_xmu);
    if (!ctx->xb) ctx->xb = new XBufs();
    return *static_cast<XBufs *>(ctx->xb);
}

void release_bufs(XBufs &B) {
    for (DevBuf *d : {&B.items, &B.work, &B.core, &B.lit, &B.copies, &B.out, &B.best, &B.planes, &B.misc, &B.vstart,
                      &B.heads})
        d->release();
    B.hbuf.release();
}

uint64_t flat_bound_h(uint64_t n) {
    if (n == 0) return 9;
    return 9 + 1 + 256 + 1 + 256 + 16 + 2 * (8 + (9 + 32 + 256 * 512 + 128 + 2 * n)) + 2 * n;
}
uint64_t nested_bound_h(uint64_t n) {
    const uint64_t r = n ? 9 + 32 + 256 * 512 + 128 + 2 * n : 9;
    const uint64_t f = flat_bound_h(n);
    return r > f ? r : f;
}

}  // namespace

void fqxv::x_release(fqxv_rans_ctx *ctx) {
    if (!ctx || !ctx->xb) return;
    XBufs *B = static_cast<XBufs *>(ctx->xb);
    release_bufs(*B);
    delete B;
    ctx->xb = nullptr;
}

extern "C" {

uint64_t fqxv_rans_x_stream_bound(uint64_t n) {
    if (n == 0) return 9;
    uint64_t st = 9 + 32;
    for (int j = 0; j < 4; j++) st += nested_bound_h((n + 3 - j) / 4);
    const uint64_t a = nested_bound_h(n);
    return a > st ? a : st;
}

uint64_t fqxv_rans_x_encode_bound(const fqxv_rans_span *blocks, size_t nblocks) {
    uint64_t b = 0;
    for (size_t i = 0; i < nblocks; i++) b += fqxv_rans_x_stream_bound(blocks[i].length);
    return b;
}

int fqxv_rans_x_encode_batch(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *blocks, size_t nblocks,
                             int flags, uint8_t *d_dst, uint64_t dst_cap, fqxv_rans_span *out_spans,
                             int32_t *out_choice) {
    if (!ctx || !out_spans || (nblocks && (!blocks || !d_dst))) return FQXV_RANS_E_INVALID_ARG;
    if (flags != FQXV_X_BEST && (flags & ~FQXV_X_ALL)) return FQXV_RANS_E_INVALID_ARG;
    if (nblocks == 0) return FQXV_RANS_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    DeviceGuard dg(ctx->device);
    XBufs &B = xbufs(ctx);
    std::vector<Span> items(nblocks);
    for (size_t i = 0; i < nblocks; i++) items[i] = Span{blocks[i].offset, blocks[i].length};
    std::vector<Span> res;
    std::vector<int32_t> choice(nblocks, flags);
    const uint8_t *arena = nullptr;
    int st;
    if (flags == FQXV_X_BEST) {
        st = encode_best(ctx, B, d_src, items, false, B.best, res, choice);
        arena = B.best.as<uint8_t>();
    } else if (flags & FQXV_X_STRIPE) {
        st = encode_stripe(ctx, B, d_src, items, flags, B.best, res);
        arena = B.best.as<uint8_t>();
    } else {
        st = encode_flat(ctx, B, d_src, items, flags, B.best, res);
        arena = B.best.as<uint8_t>();
        for (size_t i = 0; i < nblocks; i++)
            if (res[i].len == kNone) return FQXV_RANS_E_INVALID_ARG;  // PACK over more than 16 symbols
    }
    if (st) return st;
    std::vector<XCopy> cps;
    uint64_t o = 0;
    for (size_t i = 0; i < nblocks; i++) {
        out_spans[i].offset = o;
        out_spans[i].length = res[i].len;
        cps.push_back(XCopy{res[i].off, o, res[i].len});
        o += res[i].len;
        if (out_choice) out_choice[i] = choice[i];
    }
    if (o > dst_cap) return FQXV_RANS_E_DST_TOO_SMALL;
    st = run_copies(ctx, B, arena, d_dst, cps);
    if (st) return st;
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->timer.collect();
    return FQXV_RANS_OK;
}

int fqxv_rans_x_decode_batch(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *blocks, size_t nblocks,
                             uint8_t *d_dst, const fqxv_rans_span *out_spans, uint64_t *out_lens, int32_t *status) {
    if (!ctx || (nblocks && (!blocks || !out_spans || !d_dst))) return FQXV_RANS_E_INVALID_ARG;
    if (nblocks == 0) return FQXV_RANS_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    DeviceGuard dg(ctx->device);
    cudaStream_t s = ctx->stream;
    XBufs &B = xbufs(ctx);
    std::vector<XNode> nodes(nblocks);
    for (size_t i = 0; i < nblocks; i++) {
        nodes[i].src_off = blocks[i].offset;
        nodes[i].len = blocks[i].length;
        nodes[i].arena = 0;
        nodes[i].out_off = out_spans[i].offset;
        nodes[i].cap = out_spans[i].length;
    }
    // parse level by level (STRIPE planes are nodes of the next level)
    size_t lo = 0;
    uint64_t plane_bytes = 0;
    while (lo < nodes.size()) {
        const size_t hi = nodes.size();
        std::vector<Span> at;
        for (size_t k = lo; k < hi; k++) at.push_back(Span{nodes[k].src_off, nodes[k].len});
        std::vector<uint8_t> heads;
        int st = gather_heads(ctx, B, d_src, at, heads);
        if (st) return st;
        std::vector<XNode> kids;
        for (size_t k = lo; k < hi; k++) {
            if (nodes[k].arena == 1) {
                nodes[k].out_off = plane_bytes;
                plane_bytes += nodes[k].cap;
            }
            parse_node(nodes[k], heads.data() + (k - lo) * kHead, kids, hi, (int)k);
        }
        nodes.insert(nodes.end(), kids.begin(), kids.end());
        lo = hi;
    }
    // core headers: the first core right after the metadata, the second after the first
    for (int c = 0; c < 2; c++) {
        std::vector<Span> at;
        std::vector<size_t> who;
        for (size_t k = 0; k < nodes.size(); k++) {
            XNode &N = nodes[k];
            if (N.kind != 1 || N.status || c >= N.ncore || (c == 1 && N.cerr[0])) continue;
            if (c == 1) N.core_at[1] = N.core_at[0] + ((N.flags & FQXV_X_CAT) ? N.arr_len[0] : 8 + N.core_len[0]);
            const uint64_t p = N.core_at[c];
            who.push_back(k);
            at.push_back(Span{N.src_off + std::min(N.len, p), N.len - std::min(N.len, p)});
        }
        std::vector<uint8_t> heads;
        int st = gather_heads(ctx, B, d_src, at, heads);
        if (st) return st;
        for (size_t q = 0; q < who.size(); q++) {
            XNode &N = nodes[who[q]];
            const uint64_t p = N.core_at[c];
            if (N.flags & FQXV_X_CAT) {
                if (p > N.len || N.len - p < N.arr_len[c]) N.cerr[c] = FQXV_RANS_E_TRUNCATED;
                N.core_len[c] = N.arr_len[c];
                continue;
            }
            uint64_t cl = 0;
            const uint64_t avail = p > N.len ? 0 : std::min<uint64_t>(kHead, N.len - p);
            N.cerr[c] = check_core(heads.data() + q * kHead, avail, N.len, p, N.flags, N.arr_len[c], cl);
            N.core_len[c] = cl;
        }
    }
    // arrays in the work arena (PACK / RLE), plane buffer
    uint64_t woff = 0;
    for (auto &N : nodes) {
        if (N.kind != 1 || N.status) continue;
        if (N.flags & (FQXV_X_PACK | FQXV_X_RLE)) {
            N.arr_off[0] = woff;
            woff += align_up(N.m + 16, 16);
        }
        if (N.flags & FQXV_X_RLE) {
            N.arr_off[1] = woff;
            woff += align_up(N.nlit + 16, 16);
            N.arr_off[2] = woff;
            woff += align_up(N.nrb + 16, 16);
        }
    }
    CK(B.work.ensure(std::max<uint64_t>(woff, 16), s));
    CK(B.vstart.ensure(std::max<uint64_t>(woff * 8, 16), s));
    CK(B.planes.ensure(std::max<uint64_t>(plane_bytes, 16), s));
    uint8_t *arenas[3] = {d_dst, B.planes.as<uint8_t>(), B.work.as<uint8_t>()};
    // where core c of node N decodes to: (arena, offset)
    auto core_dst = [&](const XNode &N, int c, int &ar, uint64_t &off) {
        if (N.flags & FQXV_X_RLE) {
            ar = 2;
            off = N.arr_off[1 + c];
        } else if (N.flags & FQXV_X_PACK) {
            ar = 2;
            off = N.arr_off[0];
        } else {
            ar = N.arena;
            off = N.out_off;
        }
    };
    // reference streams and 32-state cores: the batched decoder, one call per output arena
    for (int ar = 0; ar < 3; ar++) {
        std::vector<fqxv_rans_span> sp, os;
        std::vector<std::pair<size_t, int>> who;  // node, core (-1: the whole reference stream)
        for (size_t k = 0; k < nodes.size(); k++) {
            XNode &N = nodes[k];
            if (N.status) continue;
            if (N.kind == 0 && N.arena == ar) {
                sp.push_back(fqxv_rans_span{N.src_off, N.len});
                os.push_back(fqxv_rans_span{N.out_off, N.cap});
                who.emplace_back(k, -1);
            } else if (N.kind == 1 && !(N.flags & (FQXV_X_CAT | FQXV_X_N4))) {
                for (int c = 0; c < N.ncore && !N.cerr[c]; c++) {
                    int a;
                    uint64_t off;
                    core_dst(N, c, a, off);
                    if (a != ar) continue;
                    sp.push_back(fqxv_rans_span{N.src_off + N.core_at[c] + 8, N.core_len[c]});
                    os.push_back(fqxv_rans_span{off, N.arr_len[c]});
                    who.emplace_back(k, c);
                }
            }
        }
        if (sp.empty()) continue;
        std::vector<uint64_t> lens(sp.size());
        std::vector<int32_t> sts(sp.size());
        const int st = decode_batch_locked(ctx, d_src, sp.data(), sp.size(), UINT64_MAX, arenas[ar], os.data(),
                                           lens.data(), sts.data());
        if (st && (st < 1 || st > 8) && st != FQXV_RANS_E_TIMEOUT) return st;
        for (size_t q = 0; q < who.size(); q++) {
            XNode &N = nodes[who[q].first];
            if (who[q].second < 0) {
                N.status = sts[q];
                if (!sts[q]) N.n = lens[q];
            } else {
                N.dstat[who[q].second] = sts[q];
            }
        }
    }
    // 4-state cores and raw (CAT) cores
    for (int ar = 0; ar < 3; ar++) {
        std::vector<XN4Dec> jobs;
        std::vector<size_t> who;
        uint64_t kmax_all = 0;
        std::vector<XCopy> cps;
        uint64_t scr = 0;
        for (size_t k = 0; k < nodes.size(); k++) {
            XNode &N = nodes[k];
            if (N.kind != 1 || N.status) continue;
            for (int c = 0; c < N.ncore && !N.cerr[c]; c++) {
                int a;
                uint64_t off;
                core_dst(N, c, a, off);
                if (a != ar) continue;
                if (N.flags & FQXV_X_CAT) {
                    cps.push_back(XCopy{N.src_off + N.core_at[c], off, N.arr_len[c]});
                } else if (N.flags & FQXV_X_N4) {
                    XN4Dec J = {};
                    J.src_off = N.src_off + N.core_at[c] + 8;
                    J.len = N.core_len[c];
                    J.dst_off = off;
                    J.cap = N.arr_len[c];
                    J.scratch_off = scr;
                    // rows for every table the core can hold (41 + 512 K bytes for K tables)
                    const uint64_t kmax = (N.flags & FQXV_X_ORDER1)
                                              ? std::min<uint64_t>(256, N.core_len[c] > 41 ? (N.core_len[c] - 41) / 512 : 0)
                                              : 1;
                    scr += std::max<uint64_t>(kmax, 1) * kN4Row;
                    kmax_all = std::max<uint64_t>(kmax_all, std::max<uint64_t>(kmax, 1));
                    jobs.push_back(J);
                    who.push_back(k * 2 + (size_t)c);
                }
            }
        }
        int st = run_copies(ctx, B, d_src, arenas[ar], cps);
        if (st) return st;
        if (jobs.empty()) continue;
        CK(B.core.ensure(std::max<uint64_t>(scr, 16), s));
        CK(B.items.ensure(jobs.size() * sizeof(XN4Dec), s));
        CK(cudaStreamSynchronize(s));
        CK(cudaMemcpyAsync(B.items.p, jobs.data(), jobs.size() * sizeof(XN4Dec), cudaMemcpyHostToDevice, s));
        {
            cudaEvent_t xt_ = ctx->timer.begin(s);
            // rows of up to kN4SmemRows tables per core in shared memory
            const int ksm = (int)std::min<uint64_t>(kmax_all, kN4SmemRows);
            ensure_n4_attr();
            x_n4_decode_kernel<<<(int)std::min<size_t>(jobs.size(), (size_t)ctx->sms * 4), 256, ksm * kN4Row, s>>>(
                d_src, B.items.as<XN4Dec>(), (int)jobs.size(), B.core.as<uint8_t>(), arenas[ar], ksm);
            ctx->timer.end(kStXDecode, xt_, s);
        }
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(jobs.data(), B.items.p, jobs.size() * sizeof(XN4Dec), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        for (size_t q = 0; q < jobs.size(); q++) nodes[who[q] / 2].dstat[who[q] % 2] = jobs[q].status;
    }
    CK(cudaStreamSynchronize(s));
    // a node's status so far: the first of its core checks and decodes
    for (auto &N : nodes) {
        if (N.kind != 1 || N.status) continue;
        for (int c = 0; c < N.ncore && !N.status; c++) N.status = N.cerr[c] ? N.cerr[c] : N.dstat[c];
    }
    // inverse RLE into A, then A (PACK: unpacked) into the output
    {
        std::vector<XUnrle> jobs;
        std::vector<size_t> who;
        for (size_t k = 0; k < nodes.size(); k++) {
            XNode &N = nodes[k];
            if (N.kind != 1 || N.status || !(N.flags & FQXV_X_RLE)) continue;
            XUnrle J = {};
            J.lit_off = N.arr_off[1];
            J.nlit = N.nlit;
            J.rb_off = N.arr_off[2];
            J.nrb = N.nrb;
            J.out_off = N.arr_off[0];
            J.m = N.m;
            std::memcpy(J.runbits, N.runbits, sizeof J.runbits);
            jobs.push_back(J);
            who.push_back(k);
        }
        if (!jobs.empty()) {
            CK(B.items.ensure(jobs.size() * sizeof(XUnrle), s));
            CK(cudaMemcpyAsync(B.items.p, jobs.data(), jobs.size() * sizeof(XUnrle), cudaMemcpyHostToDevice, s));
            {
                cudaEvent_t xt_ = ctx->timer.begin(s);
                x_unrle_kernel<<<(int)std::min<size_t>(jobs.size(), (size_t)ctx->sms * 2), kXThreads, 0, s>>>(
                    B.work.as<uint8_t>(), B.items.as<XUnrle>(), (int)jobs.size(), B.vstart.as<uint64_t>());
                ctx->timer.end(kStXDecode, xt_, s);
            }
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(jobs.data(), B.items.p, jobs.size() * sizeof(XUnrle), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            for (size_t q = 0; q < jobs.size(); q++)
                if (jobs[q].status) nodes[who[q]].status = jobs[q].status;
        }
    }
    for (int ar = 0; ar < 2; ar++) {
        std::vector<XUnpack> jobs;
        std::vector<size_t> who;
        std::vector<XCopy> cps;
        for (size_t k = 0; k < nodes.size(); k++) {
            XNode &N = nodes[k];
            if (N.kind != 1 || N.status || N.arena != ar) continue;
            if (N.flags & FQXV_X_PACK) {
                XUnpack J = {};
                J.a_off = N.arr_off[0];
                J.out_off = N.out_off;
                J.n = N.n;
                J.nsym = N.nsym;
                std::memcpy(J.syms, N.syms, 16);
                jobs.push_back(J);
                who.push_back(k);
            } else if (N.flags & FQXV_X_RLE) {
                cps.push_back(XCopy{N.arr_off[0], N.out_off, N.n});
            }
        }
        int st = run_copies(ctx, B, B.work.as<uint8_t>(), arenas[ar], cps);
        if (st) return st;
        if (jobs.empty()) continue;
        CK(B.items.ensure(jobs.size() * sizeof(XUnpack), s));
        CK(cudaStreamSynchronize(s));
        CK(cudaMemcpyAsync(B.items.p, jobs.data(), jobs.size() * sizeof(XUnpack), cudaMemcpyHostToDevice, s));
        {
            cudaEvent_t xt_ = ctx->timer.begin(s);
            x_unpack_kernel<<<(int)std::min<size_t>(jobs.size(), (size_t)ctx->sms * 4), 256, 0, s>>>(
                B.work.as<uint8_t>(), arenas[ar], B.items.as<XUnpack>(), (int)jobs.size());
            ctx->timer.end(kStXDecode, xt_, s);
        }
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(jobs.data(), B.items.p, jobs.size() * sizeof(XUnpack), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        for (size_t q = 0; q < jobs.size(); q++)
            if (jobs[q].status) nodes[who[q]].status = jobs[q].status;
    }
    // STRIPE, deepest level first (a node's planes are one level below it):
    // one launch per level, into the caller's arena at level 0 and into the
    // plane buffer below
    int maxlev = 0;
    for (auto &N : nodes) maxlev = std::max(maxlev, N.level);
    for (int lev = maxlev; lev >= 0; lev--) {
        std::vector<uint64_t> oo, on, po;
        for (auto &N : nodes) {
            if (N.kind != 2 || N.status || N.level != lev) continue;
            for (int j = 0; j < 4 && !N.status; j++) {
                if (N.child[j] == -2) {
                    N.status = FQXV_RANS_E_TRUNCATED;
                    break;
                }
                const XNode &C = nodes[N.child[j]];
                if (C.status) N.status = C.status;
                else if (C.n != C.cap) N.status = FQXV_RANS_E_X_MALFORMED;
            }
            if (N.status) continue;
            oo.push_back(N.out_off);
            on.push_back(N.n);
            for (int j = 0; j < 4; j++) po.push_back(nodes[N.child[j]].out_off);
        }
        if (oo.empty()) continue;
        const size_t k = oo.size();
        CK(B.misc.ensure(6 * k * 8 + 16, s));
        CK(cudaStreamSynchronize(s));
        uint64_t *dm = B.misc.as<uint64_t>();
        CK(cudaMemcpyAsync(dm, oo.data(), k * 8, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(dm + k, on.data(), k * 8, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(dm + 2 * k, po.data(), 4 * k * 8, cudaMemcpyHostToDevice, s));
        {
            cudaEvent_t xt_ = ctx->timer.begin(s);
            x_unstripe_kernel<<<(int)std::min<size_t>(k, (size_t)ctx->sms * 4), 256, 0, s>>>(
                B.planes.as<uint8_t>(), arenas[lev == 0 ? 0 : 1], dm, dm + k, dm + 2 * k, (int)k);
            ctx->timer.end(kStXDecode, xt_, s);
        }
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(s));
    ctx->timer.collect();
    int first = FQXV_RANS_OK;
    for (size_t i = 0; i < nblocks; i++) {
        const XNode &N = nodes[i];
        if (status) status[i] = N.status;
        if (out_lens) out_lens[i] = N.status ? 0 : N.n;
        if (N.status && !first) first = N.status;
    }
    return first;
}

}  // extern "C"
