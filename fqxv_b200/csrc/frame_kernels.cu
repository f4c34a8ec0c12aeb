// CRC-32C (crates/fqxv/src/crc.rs) and container block frames
// (crates/fqxv/src/container/block.rs) on B200.
//
// A CRC-32C pass covers a list of targets (byte ranges). Each target is cut
// into pieces at multiples of a power-of-two piece size; one warp computes a
// piece's CRC contribution and XORs it, shifted to the target's end, into the
// target's result (CRC-32C is linear over GF(2), so pieces combine in any
// order). The plan kernel (one warp per target) writes the piece list and the
// target's init/xor-out term; the piece kernel is persistent (one 1024-thread
// CTA per SM, warps pull pieces from a counter).
//
// Inside a piece, lane l owns the 4-byte word l of every 128-byte line. Its
// state advances as s <- Z^128(s ^ w), Z^k being "append k zero bytes"
// (multiplication by x^(8k) mod P). Z^128 is linear, so it is four byte
// lookups; the tables are replicated once per lane (lane l reads column l)
// so the lookups of a warp never share a bank. After its last word a lane
// shifts its state to the piece end by one GF(2) multiplication; a warp XOR
// reduction gives the piece's raw CRC.
//
// Polynomial arithmetic is in the reflected representation of crc.rs: bit 31
// of a word is the coefficient of x^0, bit 0 of x^31; multiplying by x is a
// right shift that folds the reflected polynomial 0x82F63B78 back in.
#include <algorithm>
#include <mutex>

#include "frame_internal.cuh"

namespace fqxv {
namespace {

constexpr uint32_t kPoly = 0x82F63B78u;
constexpr uint32_t kOne = 0x80000000u;  // the polynomial 1
constexpr int kZMax = 132;              // Z^r multipliers kept for r < kZMax

// a(x) * b(x) mod P, reflected.
__host__ __device__ constexpr uint32_t gf_mul_c(uint32_t a, uint32_t b) {
    uint32_t p = 0;
    for (int i = 31; i >= 0; i--) {
        if ((a >> i) & 1u) p ^= b;
        b = (b >> 1) ^ ((b & 1u) ? kPoly : 0u);
    }
    return p;
}

struct CrcConsts {
    uint32_t z[kZMax];     // x^(8 r) mod P
};

constexpr CrcConsts make_consts() {
    CrcConsts c{};
    c.z[0] = kOne;
    for (int r = 1; r < kZMax; r++) c.z[r] = gf_mul_c(c.z[r - 1], kOne >> 8);
    return c;
}

__constant__ CrcConsts c_crc = make_consts();

// t[k][b] = x^(8 b 256^k) mod P: x^(8 n) for a 64-bit n is the product of
// one entry per nonzero byte of n.
struct PowTables {
    uint32_t t[8][256];
};

constexpr PowTables make_pow_tables() {
    PowTables p{};
    uint32_t base = kOne >> 8;  // x^8
    for (int k = 0; k < 8; k++) {
        p.t[k][0] = kOne;
        for (int b = 1; b < 256; b++) p.t[k][b] = gf_mul_c(p.t[k][b - 1], base);
        for (int i = 0; i < 8; i++) base = gf_mul_c(base, base);  // x^(8 256^(k+1))
    }
    return p;
}

__device__ const PowTables c_powb = make_pow_tables();

__device__ __forceinline__ uint32_t gf_mul(uint32_t a, uint32_t b) {
    uint32_t p = 0;
#pragma unroll
    for (int i = 31; i >= 0; i--) {
        p ^= b & (0u - ((a >> i) & 1u));
        b = (b >> 1) ^ (kPoly & (0u - (b & 1u)));
    }
    return p;
}

// x^(8 n) mod P (n zero bytes appended).
__device__ __forceinline__ uint32_t pow8(uint64_t n) {
    uint32_t f = kOne;
    for (int k = 0; k < 8 && n; k++, n >>= 8) {
        const uint32_t b = (uint32_t)(n & 0xFFu);
        if (b) f = gf_mul(f, __ldg(&c_powb.t[k][b]));
    }
    return f;
}

// ---- plan: pieces and init terms ------------------------------------------
// One warp per target. A target's pieces are cut at multiples of the piece
// size in the address space the piece kernel aligns its lines to (the
// destination for a frame copy, the source otherwise), so a destination word
// is never written by two warps. Result init: the CRC of a target of n bytes
// is raw(bytes) ^ Z^n(~0) ^ ~0 (crc.rs:48-66: register preset to ~0, final
// xor ~0), and the second and third terms are written here.
__global__ void crc_plan_kernel(FrameJob *job, CrcTarget *targets, CrcPiece *pieces, uint32_t *crc_out,
                                uint64_t align_base, int by_dst) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    const uint32_t n = job->ntargets;
    const int psh = job->piece_shift;
    for (uint32_t t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < n; t += warps) {
        const CrcTarget T = targets[t];
        if (lane == 0) crc_out[t] = gf_mul(0xFFFFFFFFu, pow8(T.len)) ^ 0xFFFFFFFFu;
        if (T.len == 0) continue;
        const uint64_t a0 = (align_base + (by_dst ? T.dst_off : T.src_off)) & ((1ull << psh) - 1);
        const uint64_t np = ((a0 + T.len - 1) >> psh) + 1;
        for (uint64_t j = lane; j < np; j += 32) {
            const uint64_t lo = j == 0 ? 0 : (j << psh) - a0;
            const uint64_t hi0 = ((j + 1) << psh) - a0;
            const uint64_t hi = hi0 < T.len ? hi0 : T.len;
            CrcPiece pc;
            pc.src = T.src_off + lo;
            pc.dst = T.dst_off + lo;
            pc.len = (uint32_t)(hi - lo);
            pc.target = t;
            pc.mult = pow8(T.len - hi);  // shifts the piece's CRC to the target's end
            pc.pad = 0;
            pieces[T.piece_base + j] = pc;
        }
    }
}

// ---- the piece kernel -------------------------------------------------------

// Word of a line masked to the bytes of [lo, hi); y is its address.
__device__ __forceinline__ uint32_t mask_word(uint32_t w, uint64_t y, uint64_t lo, uint64_t hi) {
    if (y + 4 <= lo || y >= hi) return 0;
    if (y < lo) w &= 0xFFFFFFFFu << (8 * (uint32_t)(lo - y));
    if (y + 4 > hi) w &= 0xFFFFFFFFu >> (8 * (uint32_t)(y + 4 - hi));
    return w;
}

__device__ __forceinline__ uint32_t ld_stream(const uint32_t *p) { return __ldcs(p); }

// The 4-byte word at aligned source address a, or 0 when it holds no byte of
// the source range [lo, hi) (so nothing outside the range is ever read).
__device__ __forceinline__ uint32_t ld_guard(uint64_t a, uint64_t lo, uint64_t hi) {
    return (a + 4 > lo && a < hi) ? ld_stream(reinterpret_cast<const uint32_t *>(a)) : 0u;
}

// Stores the bytes of word w (destination address y) that fall in [lo, hi).
__device__ __forceinline__ void st_masked(uint32_t w, uint64_t y, uint64_t lo, uint64_t hi) {
    if (y >= lo && y + 4 <= hi) {
        __stcs(reinterpret_cast<uint32_t *>(y), w);
        return;
    }
#pragma unroll
    for (int b = 0; b < 4; b++)
        if (y + b >= lo && y + b < hi) *reinterpret_cast<uint8_t *>(y + b) = (uint8_t)(w >> (8 * b));
}

// Shared memory: the four Z^128 byte tables, replicated once per lane, then
// the Z^r multipliers. Entry b of table k for lane l sits at byte
//   (k & 1) * 64 KiB + b * 256 + (k >> 1) * 128 + l * 4,
// so a warp's 32 lookups hit 32 banks, and the address of a lookup is one
// byte permute: [l * 4, byte k of x, 0, 0] plus an immediate table base.
constexpr uint32_t kTabWords = 4 * 256 * 32;
constexpr uint32_t kPieceSmem = (kTabWords + kZMax) * 4;

struct LaneTables {
    const uint8_t *base;  // shared memory base of the tables
    uint32_t lane4;       // l * 4
    __device__ __forceinline__ uint32_t at(uint32_t off) const {
        return *reinterpret_cast<const uint32_t *>(base + off);
    }
    __device__ __forceinline__ uint32_t step(uint32_t x) const {
        const uint32_t a0 = __byte_perm(x, lane4, 0x5504);  // byte 0 of x
        const uint32_t a1 = __byte_perm(x, lane4, 0x5514);
        const uint32_t a2 = __byte_perm(x, lane4, 0x5524);
        const uint32_t a3 = __byte_perm(x, lane4, 0x5534);
        return at(a0) ^ at(a1 + 65536u) ^ at(a2 + 128u) ^ at(a3 + 65536u + 128u);
    }
};

__device__ __forceinline__ uint32_t tab_offset(uint32_t k, uint32_t b, uint32_t lane) {
    return (k & 1u) * 65536u + b * 256u + (k >> 1) * 128u + lane * 4u;
}

__device__ void build_tables(uint32_t *smem) {
    const int lane = threadIdx.x & 31;
    uint8_t *sb = reinterpret_cast<uint8_t *>(smem);
    // entry e = 256 k + b of table k: (b << 8k) * x^(8 * 128); a warp computes
    // 32 consecutive entries, one a lane, and writes them lane by lane
    for (uint32_t base = threadIdx.x & ~31u; base < 1024; base += blockDim.x) {
        const uint32_t e = base + lane;
        const uint32_t v = gf_mul((e & 0xFFu) << (8 * (e >> 8)), c_crc.z[128]);
        for (int j = 0; j < 32; j++) {
            const uint32_t x = __shfl_sync(0xFFFFFFFFu, v, j);
            const uint32_t ej = base + j;
            *reinterpret_cast<uint32_t *>(sb + tab_offset(ej >> 8, ej & 0xFFu, lane)) = x;
        }
    }
    for (uint32_t i = threadIdx.x; i < kZMax; i += blockDim.x) smem[kTabWords + i] = c_crc.z[i];
}

__device__ __forceinline__ CrcPiece load_piece(const CrcPiece *p) {
    const uint4 a = __ldg(reinterpret_cast<const uint4 *>(p));
    const uint4 b = __ldg(reinterpret_cast<const uint4 *>(p) + 1);
    CrcPiece c;
    c.src = ((uint64_t)a.y << 32) | a.x;
    c.dst = ((uint64_t)a.w << 32) | a.z;
    c.len = b.x;
    c.target = b.y;
    c.mult = b.z;
    c.pad = b.w;
    return c;
}

// Pieces are dealt to warps round-robin (they are all of the piece size but
// the targets' ends); a warp prefetches its next piece's record while it
// works on the current one, and keeps the loads of the next U lines in
// flight while it folds in the current U.
template <bool COPY, int U, int THREADS>
__global__ void __launch_bounds__(THREADS, 1)
    crc_piece_kernel(const uint8_t *src, uint8_t *dst, const FrameJob *job, const CrcPiece *pieces,
                     uint32_t *crc_out) {
    extern __shared__ uint32_t smem[];
    build_tables(smem);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const LaneTables G{reinterpret_cast<const uint8_t *>(smem), 4u * lane};
    const uint32_t *sZ = smem + kTabWords;
    const uint32_t npieces = job->npieces;
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
    uint32_t pi = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    CrcPiece pc{};
    if (pi < npieces) pc = load_piece(pieces + pi);
    while (pi < npieces) {
        const uint32_t pn = pi + nwarps;
        CrcPiece nx{};
        if (pn < npieces) nx = load_piece(pieces + pn);
        // Line grid: aligned on the destination for a copy, else the source.
        const uint64_t s0 = reinterpret_cast<uint64_t>(src + pc.src);
        const uint64_t d0 = COPY ? reinterpret_cast<uint64_t>(dst + pc.dst) : s0;
        const uint64_t lo = d0, hi = d0 + pc.len;
        const uint64_t Ya = lo & ~3ull;
        const uint32_t nlines = (uint32_t)((hi - Ya + 127) >> 7);
        const uint64_t y0 = Ya + 4 * lane;
        const uint32_t last = (nlines >= 2 && y0 + 128ull * (nlines - 1) >= hi) ? nlines - 2 : nlines - 1;
        // copy: source address of destination byte y is y + delta; a
        // destination word is bytes sh.. of two aligned source words
        const uint64_t delta = s0 - d0;
        const uint32_t sh = COPY ? (uint32_t)((Ya + delta) & 3) : 0;
        const uint64_t as0 = Ya + delta - sh + 4 * lane;  // lane's aligned source word, line 0
        const uint64_t slo = s0, shi = s0 + pc.len;

        // One line's word for this lane: loaded (guarded when `edge`),
        // realigned for a copy, masked to the piece, and stored for a copy.
        auto word = [&](uint32_t m, bool edge) -> uint32_t {
            const uint64_t y = y0 + 128ull * m;
            if (!COPY) {
                const uint32_t w = edge ? ld_guard(y, lo, hi) : ld_stream(reinterpret_cast<const uint32_t *>(y));
                return edge ? mask_word(w, y, lo, hi) : w;
            }
            const uint64_t a = as0 + 128ull * m;
            const uint32_t w0 = edge ? ld_guard(a, slo, shi) : ld_stream(reinterpret_cast<const uint32_t *>(a));
            uint32_t w = w0;
            if (sh) {
                uint32_t w1 = __shfl_down_sync(0xFFFFFFFFu, w0, 1);
                if (lane == 31) w1 = ld_guard(a + 4, slo, shi);
                w = __funnelshift_r(w0, w1, 8 * sh);
            }
            if (edge) {
                w = mask_word(w, y, lo, hi);
                st_masked(w, y, lo, hi);
            } else {
                __stcs(reinterpret_cast<uint32_t *>(y), w);
            }
            return w;
        };

        uint32_t s = 0;
        {
            const uint32_t x = word(0, true);
            s = last == 0 ? x : G.step(x);
        }
        // Lines [1, nlines - 2) are whole and no lane's last: loads of the
        // next U lines are issued before the current U are folded in.
        const uint32_t mid_end = nlines >= 3 ? nlines - 2 : 1;
        uint32_t m = 1;
        const uint32_t *q = reinterpret_cast<const uint32_t *>(COPY ? as0 : y0);
        uint32_t *o = reinterpret_cast<uint32_t *>(y0);
        // lane 31's second source word of line j is lane 0's word of line
        // j + 1: a shuffle within a batch, one load for the batch's last line
        const bool extra = COPY && sh && lane == 31;
        uint32_t wa[U], wb[U], xa = 0, xb = 0;
        auto load = [&](uint32_t *w, uint32_t &xl, uint32_t mm) {
#pragma unroll
            for (int j = 0; j < U; j++) w[j] = ld_stream(q + 32 * (mm + j));
            if (extra) xl = ld_stream(q + 32 * (mm + U - 1) + 1);
        };
        auto fold = [&](const uint32_t *w, uint32_t xl, uint32_t mm) {
#pragma unroll
            for (int j = 0; j < U; j++) {
                uint32_t v = w[j];
                if (COPY) {
                    if (sh) {
                        uint32_t w1 = __shfl_down_sync(0xFFFFFFFFu, w[j], 1);
                        const uint32_t nx0 = j + 1 < U ? __shfl_sync(0xFFFFFFFFu, w[j + 1 < U ? j + 1 : j], 0) : xl;
                        if (lane == 31) w1 = nx0;
                        v = __funnelshift_r(w[j], w1, 8 * sh);
                    }
                    __stcs(o + 32 * (mm + j), v);
                }
                s = G.step(s ^ v);
            }
        };
        if (m + U <= mid_end) load(wa, xa, m);
        while (m + U <= mid_end) {
            const bool nb = m + 2 * U <= mid_end;
            if (nb) load(wb, xb, m + U);
            fold(wa, xa, m);
            m += U;
            if (!nb) break;
            const bool na = m + 2 * U <= mid_end;
            if (na) load(wa, xa, m + U);
            fold(wb, xb, m);
            m += U;
            if (!na) break;
        }
        for (; m < mid_end; m++) s = G.step(s ^ word(m, false));
        if (nlines >= 3) {
            const uint32_t x = s ^ word(nlines - 2, false);
            s = last == nlines - 2 ? x : G.step(x);
        }
        if (nlines >= 2) {
            // every lane takes part (the copy's shuffle); only lanes whose
            // last word is here fold it in
            const uint32_t w = word(nlines - 1, true);
            if (last == nlines - 1) s ^= w;
        }
        // Shift to the piece end: the lane's last word starts r bytes before it.
        const uint64_t ylast = y0 + 128ull * last;
        const uint64_t rr = hi > ylast ? hi - ylast : 0;
        const uint32_t r = rr < (uint64_t)(kZMax - 1) ? (uint32_t)rr : (uint32_t)(kZMax - 1);
        uint32_t raw = s ? gf_mul(s, sZ[r]) : 0u;
#pragma unroll
        for (int o2 = 16; o2; o2 >>= 1) raw ^= __shfl_xor_sync(0xFFFFFFFFu, raw, o2);
        if (lane == 0 && raw) atomicXor(&crc_out[pc.target], gf_mul(raw, pc.mult));
        pi = pn;
        pc = nx;
    }
}

// ---- frame heads ------------------------------------------------------------
// block.rs:125-128: [4 "FQXB"][u64 payload_len][u32 crc32c(payload)] before
// each payload (dst_off is the payload's place; the head takes the 16 bytes
// before it), and when term_off != ~0 the zero-length terminator frame.
__global__ void frame_heads_kernel(uint8_t *dst, const FrameJob *job, const CrcTarget *targets,
                                   const uint32_t *crc_out, uint64_t term_off) {
    const uint32_t n = job->ntargets;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t <= n; t += gridDim.x * blockDim.x) {
        uint8_t *h;
        uint64_t len;
        uint32_t crc = 0;
        if (t < n) {
            h = dst + targets[t].dst_off - kFrameHead;
            len = targets[t].len;
            crc = crc_out[t];
        } else {
            if (term_off == ~0ull) continue;
            h = dst + term_off;
            len = 0;
        }
        h[0] = 'F';
        h[1] = 'Q';
        h[2] = 'X';
        h[3] = 'B';
        for (int b = 0; b < 8; b++) h[4 + b] = (uint8_t)(len >> (8 * b));
        if (t < n)
            for (int b = 0; b < 4; b++) h[12 + b] = (uint8_t)(crc >> (8 * b));
    }
}

// ---- frame walk ---------------------------------------------------------------
// block.rs:1209-1254 applied frame after frame from offset 0. Each frame's
// place depends on the previous frame's length, so the walk is a chain:
//   1. one thread walks the first kWalkHops frames (a dependent load per hop);
//   2. if frames remain, every thread scans the rest of the buffer for the
//      frame marker "FQXB" and records each hit with the 12 bytes after it;
//   3. one CTA sorts the hits, links each to the hit where its frame ends,
//      ranks the chain from the walk's position by pointer doubling, and
//      writes the walk entries of the chain in parallel.
// Every frame start is a hit (a frame starts with the marker), so the chain
// through the hits is the serial walk's chain; a hit inside a payload is
// never reached from the chain's head. More hits than the chain kernel holds
// (or a buffer of 4 GiB or more past the head) fall back to the serial walk.
__device__ __forceinline__ uint64_t rd_le(const uint8_t *p, int n) {
    uint64_t v = 0;
    for (int i = 0; i < n; i++) v |= (uint64_t)p[i] << (8 * i);
    return v;
}

constexpr uint32_t kFrameMagic = 0x42585146u;  // "FQXB" little-endian

// The serial walk from job->walk_pos, at most max_hops loop iterations;
// returns true when the walk is over (end, terminator, failure or
// max_frames). Walk state lives in the job header.
__device__ bool serial_walk(const uint8_t *src, uint64_t len, uint32_t max_frames, FrameJob *job,
                            CrcTarget *targets, WalkEntry *walk, uint32_t max_hops) {
    uint64_t pos = job->walk_pos;
    uint32_t k = job->nframes, nt = job->ntargets;
    bool done = false;
    for (uint32_t hop = 0;; hop++) {
        if (k >= max_frames || len - pos < 4) {
            done = true;
            break;
        }
        if (hop >= max_hops) break;
        const uint64_t left = len - pos;
        const uint8_t *f = src + pos;
        int32_t st = FQXV_RANS_OK;
        uint64_t plen = 0;
        if (f[0] != 'F' || f[1] != 'Q' || f[2] != 'X' || f[3] != 'B') {
            st = FQXV_FRAME_E_BAD_SYNC;
        } else if (left < 12) {
            st = FQXV_FRAME_E_TRUNCATED;
        } else {
            plen = rd_le(f + 4, 8);
            if (plen == 0) {
                pos += kFrameTerm;
                job->terminated = 1;
                done = true;
                break;
            }
            if (plen > kMaxBlockPayload) st = FQXV_FRAME_E_TOO_LARGE;
            else if (left < kFrameHead || left - kFrameHead < plen) st = FQXV_FRAME_E_TRUNCATED;
        }
        WalkEntry e;
        if (st != FQXV_RANS_OK) {
            e.pay_off = pos;
            e.pay_len = 0;
            e.stored_crc = 0;
            e.crc = 0;
            e.status = st;
            e.target = ~0u;
            walk[k++] = e;
            done = true;
            break;
        }
        e.pay_off = pos + kFrameHead;
        e.pay_len = plen;
        e.stored_crc = (uint32_t)rd_le(f + 12, 4);
        e.crc = 0;
        e.status = FQXV_RANS_OK;
        e.target = nt;
        targets[nt++] = CrcTarget{e.pay_off, plen, 0, 0};
        walk[k++] = e;
        pos += kFrameHead + plen;
    }
    job->walk_pos = pos;
    job->nframes = k;
    job->ntargets = nt;
    job->consumed = pos;
    job->walk_done = done ? 1u : 0u;
    return done;
}

__global__ void frame_walk_kernel(const uint8_t *src, uint64_t len, uint32_t max_frames, FrameJob *job,
                                  CrcTarget *targets, WalkEntry *walk) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    job->walk_pos = 0;
    job->nframes = 0;
    job->ntargets = 0;
    job->terminated = 0;
    job->ncand = 0;
    job->cand_overflow = 0;
    job->counter = 0;
    serial_walk(src, len, max_frames, job, targets, walk, kWalkHops);
}

// Marker hits in [walk_pos, len): 16 bytes a thread, four blocks in flight.
__global__ void frame_scan_kernel(const uint8_t *src, uint64_t len, FrameJob *job, WalkCand *cand) {
    if (job->walk_done) return;
    const uint64_t lo = reinterpret_cast<uint64_t>(src) + job->walk_pos;
    const uint64_t end = reinterpret_cast<uint64_t>(src) + len;
    const uint64_t a0 = lo & ~15ull;
    const uint64_t stride = 16ull * gridDim.x * blockDim.x;
    for (uint64_t c0 = a0 + 16ull * (blockIdx.x * blockDim.x + threadIdx.x); c0 < end; c0 += 4 * stride) {
        uint4 v[4];
        uint32_t nx[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const uint64_t c = c0 + u * stride;
            if (c < end) {
                v[u] = __ldcs(reinterpret_cast<const uint4 *>(c));
                nx[u] = c + 16 < end ? __ldcs(reinterpret_cast<const uint32_t *>(c + 16)) : 0u;
            }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const uint64_t c = c0 + u * stride;
            if (c >= end) continue;
            const uint32_t w[5] = {v[u].x, v[u].y, v[u].z, v[u].w, nx[u]};
            bool any = false;
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const uint32_t x = (i & 3) ? __funnelshift_r(w[i >> 2], w[(i >> 2) + 1], 8 * (i & 3)) : w[i >> 2];
                any |= x == kFrameMagic;
            }
            if (!any) continue;
            for (int i = 0; i < 16; i++) {
                const uint32_t x = (i & 3) ? __funnelshift_r(w[i >> 2], w[(i >> 2) + 1], 8 * (i & 3)) : w[i >> 2];
                const uint64_t p = c + i;
                if (x == kFrameMagic && p >= lo && p + 4 <= end) {
                    const uint32_t idx = atomicAdd(&job->ncand, 1u);
                    if (idx >= kChainMax) {
                        job->cand_overflow = 1;
                        continue;
                    }
                    const uint8_t *f = reinterpret_cast<const uint8_t *>(p);
                    WalkCand wc;
                    wc.pos = p - reinterpret_cast<uint64_t>(src);
                    wc.plen = p + 12 <= end ? rd_le(f + 4, 8) : 0;
                    wc.crc = p + 16 <= end ? (uint32_t)rd_le(f + 12, 4) : 0;
                    wc.pad = 0;
                    cand[idx] = wc;
                }
            }
        }
    }
}

// Node kinds of the chain kernel.
enum : uint8_t { kNodeNext, kNodeEnd, kNodeBadNext, kNodeTerm, kNodeTrunc, kNodeTooLarge };
constexpr uint16_t kNone = 0xFFFF;

__global__ void __launch_bounds__(1024, 1)
    frame_chain_kernel(const uint8_t *src, uint64_t len, uint32_t max_frames, FrameJob *job, CrcTarget *targets,
                       WalkEntry *walk, const WalkCand *cand) {
    if (job->walk_done) return;
    const uint32_t nc = job->ncand;
    const uint64_t base = job->walk_pos;
    const uint32_t k0 = job->nframes, nt0 = job->ntargets;
    if (job->cand_overflow || nc > kChainMax || len - base >= (1ull << 32)) {
        if (threadIdx.x == 0) serial_walk(src, len, max_frames, job, targets, walk, 0xFFFFFFFFu);
        return;
    }
    const uint32_t span = (uint32_t)(len - base);  // bytes from the head
    extern __shared__ uint64_t csm[];
    uint64_t *key = csm;                                            // [kChainMax] (pos << 13) | hit index
    uint32_t *plen = reinterpret_cast<uint32_t *>(key + kChainMax);  // [kChainMax] (> 2^31: too large)
    uint32_t *crc = plen + kChainMax;                               // [kChainMax]
    uint16_t *succ = reinterpret_cast<uint16_t *>(crc + kChainMax);  // [kChainMax]
    uint16_t *jmp = succ + kChainMax;                                // [kChainMax]
    uint16_t *rank = jmp + kChainMax;                                // [kChainMax]
    uint8_t *kind = reinterpret_cast<uint8_t *>(rank + kChainMax);   // [kChainMax]
    __shared__ uint32_t s_len, s_head, s_last, s_nok;
    __shared__ unsigned long long s_cut;
    const uint32_t tid = threadIdx.x, nth = blockDim.x;
    uint32_t n2 = 1;
    while (n2 < nc) n2 <<= 1;
    for (uint32_t i = tid; i < n2; i += nth)
        key[i] = i < nc ? ((cand[i].pos - base) << 13) | i : ~0ull;
    if (tid == 0) {
        s_len = 0;
        s_nok = 0;
        s_cut = 0;
        s_last = kNone;
    }
    __syncthreads();
    // bitonic sort of the hits by position
    for (uint32_t k = 2; k <= n2; k <<= 1)
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = tid; i < n2; i += nth) {
                const uint32_t l = i ^ j;
                if (l > i) {
                    const uint64_t a = key[i], b = key[l];
                    if (((i & k) == 0) == (a > b)) {
                        key[i] = b;
                        key[l] = a;
                    }
                }
            }
            __syncthreads();
        }
    for (uint32_t i = tid; i < nc; i += nth) {
        const WalkCand c = cand[key[i] & 0x1FFF];
        plen[i] = c.plen > kMaxBlockPayload ? (uint32_t)kMaxBlockPayload + 1 : (uint32_t)c.plen;
        crc[i] = c.crc;
    }
    __syncthreads();
    // each hit's frame and the hit where it ends
    for (uint32_t i = tid; i < nc; i += nth) {
        const uint32_t P = (uint32_t)(key[i] >> 13);
        const uint32_t left = span - P;
        uint8_t kd;
        uint16_t nx = kNone;
        if (left < 12) {
            kd = kNodeTrunc;
        } else if (plen[i] == 0) {
            kd = kNodeTerm;
        } else if (plen[i] > kMaxBlockPayload) {
            kd = kNodeTooLarge;
        } else if (left < kFrameHead || left - kFrameHead < plen[i]) {
            kd = kNodeTrunc;
        } else {
            const uint64_t np = (uint64_t)P + kFrameHead + plen[i];
            if (span - np < 4) {
                kd = kNodeEnd;
            } else {
                uint32_t a = 0, b = nc;  // first hit at or after np
                while (a < b) {
                    const uint32_t m = (a + b) >> 1;
                    if ((key[m] >> 13) < np) a = m + 1;
                    else b = m;
                }
                if (a < nc && (key[a] >> 13) == np) {
                    kd = kNodeNext;
                    nx = (uint16_t)a;
                } else {
                    kd = kNodeBadNext;
                }
            }
        }
        kind[i] = kd;
        succ[i] = nx;
        jmp[i] = nx;
        rank[i] = kNone;
    }
    __syncthreads();
    if (tid == 0) {
        s_head = (nc > 0 && (key[0] >> 13) == 0) ? 0u : kNone;
        if (s_head != kNone) rank[0] = 0;
    }
    __syncthreads();
    if (s_head == kNone) {
        // no marker at the walk's position
        if (tid == 0) {
            uint32_t k = k0;
            if (k < max_frames) {
                WalkEntry e{base, 0, 0, 0, FQXV_FRAME_E_BAD_SYNC, ~0u};
                walk[k++] = e;
            }
            job->nframes = k;
            job->consumed = base;
            job->walk_done = 1;
        }
        return;
    }
    // ranks from the head by pointer doubling: after round t every hit within
    // 2^(t+1) hops of the head is ranked and jmp is succ^(2^(t+1))
    for (uint32_t t = 0; (1u << t) < nc; t++) {
        for (uint32_t i = tid; i < nc; i += nth) {
            const uint16_t r = rank[i];
            const uint16_t j = jmp[i];
            if (r != kNone && j != kNone) rank[j] = (uint16_t)(r + (1u << t));
        }
        __syncthreads();
        uint16_t nj[kChainMax / 1024];
        uint32_t q = 0;
        for (uint32_t i = tid; i < nc; i += nth, q++) nj[q] = jmp[i] == kNone ? kNone : jmp[jmp[i]];
        __syncthreads();
        q = 0;
        for (uint32_t i = tid; i < nc; i += nth, q++) jmp[i] = nj[q];
        __syncthreads();
    }
    // the chain's length: its last hit is the ranked one with no successor
    for (uint32_t i = tid; i < nc; i += nth)
        if (rank[i] != kNone && succ[i] == kNone) {
            s_len = rank[i] + 1u;
            s_last = i;
        }
    __syncthreads();
    const uint32_t L = s_len;
    const uint32_t e = s_last;
    // frames the walk processes: hit r is read while k0 + r < max_frames
    const uint32_t lim = max_frames - k0;  // > 0 (the serial walk stopped below max_frames)
    for (uint32_t i = tid; i < nc; i += nth) {
        const uint32_t r = rank[i];
        if (r == kNone || r >= lim) continue;
        const uint32_t P = (uint32_t)(key[i] >> 13);
        const uint8_t kd = kind[i];
        if (kd == kNodeTerm) continue;
        WalkEntry we;
        if (kd == kNodeTrunc || kd == kNodeTooLarge) {
            we = WalkEntry{base + P, 0, 0, 0, kd == kNodeTrunc ? FQXV_FRAME_E_TRUNCATED : FQXV_FRAME_E_TOO_LARGE,
                           ~0u};
        } else {
            we = WalkEntry{base + P + kFrameHead, plen[i], crc[i], 0, FQXV_RANS_OK, nt0 + r};
            targets[nt0 + r] = CrcTarget{base + P + kFrameHead, plen[i], 0, 0};
            atomicAdd(&s_nok, 1u);
            if (r == lim - 1) s_cut = base + P + kFrameHead + plen[i];  // where a max_frames cut stops
        }
        walk[k0 + r] = we;
    }
    __syncthreads();
    if (tid == 0) {
        // where the walk stopped
        uint32_t k = k0 + (L < lim ? L : lim);
        uint64_t consumed;
        if (L > lim) {
            consumed = s_cut;  // cut by max_frames before the chain's end
        } else {
            const uint32_t P = (uint32_t)(key[e] >> 13);
            const uint8_t kd = kind[e];
            if (kd == kNodeTerm) {
                k -= 1;  // the terminator is not a frame
                consumed = base + P + kFrameTerm;
                job->terminated = 1;
            } else if (kd == kNodeTrunc || kd == kNodeTooLarge) {
                consumed = base + P;
            } else {
                consumed = base + P + kFrameHead + plen[e];
                if (kd == kNodeBadNext && k < max_frames) {
                    walk[k++] = WalkEntry{consumed, 0, 0, 0, FQXV_FRAME_E_BAD_SYNC, ~0u};
                }
            }
        }
        job->nframes = k;
        job->ntargets = nt0 + s_nok;
        job->consumed = consumed;
        job->walk_pos = consumed;
        job->walk_done = 1;
    }
}

// Piece size and piece bases of the job's targets: one CTA, each thread a
// run of consecutive targets (total -> piece size, counts -> block scan).
__global__ void __launch_bounds__(1024, 1)
    piece_bases_kernel(FrameJob *job, CrcTarget *targets, uint64_t align_base) {
    __shared__ unsigned long long s_sum[1024];
    __shared__ unsigned long long s_total;
    const uint32_t n = job->ntargets;
    const uint32_t tid = threadIdx.x, nth = blockDim.x;
    const uint32_t per = (n + nth - 1) / nth;
    const uint32_t lo = tid * per < n ? tid * per : n;
    const uint32_t hi = lo + per < n ? lo + per : n;
    unsigned long long t = 0;
    for (uint32_t i = lo; i < hi; i++) t += targets[i].len;
    s_sum[tid] = t;
    __syncthreads();
    for (uint32_t o = nth >> 1; o; o >>= 1) {  // total (nth is a power of two)
        if (tid < o) s_sum[tid] += s_sum[tid + o];
        __syncthreads();
    }
    if (tid == 0) s_total = s_sum[0];
    __syncthreads();
    const int psh = crc_piece_shift(s_total, kCrcPieceTarget, kCrcMinShift, kCrcMaxShift);
    unsigned long long c = 0;
    for (uint32_t i = lo; i < hi; i++) c += crc_piece_count(align_base + targets[i].src_off, targets[i].len, psh);
    s_sum[tid] = c;
    __syncthreads();
    for (uint32_t o = 1; o < nth; o <<= 1) {  // inclusive scan
        const unsigned long long v = tid >= o ? s_sum[tid - o] : 0ull;
        __syncthreads();
        s_sum[tid] += v;
        __syncthreads();
    }
    unsigned long long b = s_sum[tid] - c;
    for (uint32_t i = lo; i < hi; i++) {
        targets[i].piece_base = b;
        b += crc_piece_count(align_base + targets[i].src_off, targets[i].len, psh);
    }
    if (tid == nth - 1) {
        job->npieces = (uint32_t)s_sum[tid];
        job->piece_shift = psh;
        job->counter = 0;
    }
}

// Frames whose computed CRC differs from the stored one become CORRUPT.
__global__ void frame_verify_kernel(const FrameJob *job, WalkEntry *walk, const uint32_t *crc_out) {
    const uint32_t n = job->nframes;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        WalkEntry &e = walk[k];
        if (e.target == ~0u) continue;
        e.crc = crc_out[e.target];
        if (e.crc != e.stored_crc) e.status = FQXV_FRAME_E_CORRUPT;
    }
}

// block.rs:961-980: the three coded streams of a plain payload
// [24 digests][u32 n_reads]([u32 len][bytes]) x 3 become CRC targets 3i..3i+2;
// a payload too short for the walk is Error::Truncated.
__global__ void stream_locs_kernel(const uint8_t *src, const PayloadRef *payloads, uint32_t n, FrameJob *job,
                                   CrcTarget *targets, int32_t *status) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const PayloadRef P = payloads[i];
        const uint8_t *p = src + P.off;
        uint64_t q = 3 * 8 + 4;
        int32_t st = P.len < q ? FQXV_FRAME_E_TRUNCATED : FQXV_RANS_OK;
        for (int s = 0; s < 3; s++) {
            CrcTarget T;
            T.src_off = P.off;
            T.len = 0;
            T.dst_off = 0;
            T.piece_base = 0;
            if (st == FQXV_RANS_OK) {
                if (P.len - q < 4) {
                    st = FQXV_FRAME_E_TRUNCATED;
                } else {
                    const uint64_t m = rd_le(p + q, 4);
                    q += 4;
                    if (P.len - q < m) {
                        st = FQXV_FRAME_E_TRUNCATED;
                    } else {
                        T.src_off = P.off + q;
                        T.len = m;
                        q += m;
                    }
                }
            }
            targets[3 * i + s] = T;
        }
        if (st != FQXV_RANS_OK)
            for (int s = 0; s < 3; s++) targets[3 * i + s].len = 0;
        status[i] = st;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        job->ntargets = 3 * n;
        job->counter = 0;
    }
}

}  // namespace

// ---- launchers -------------------------------------------------------------------

// The piece kernels' dynamic shared memory limit, raised once per device
// (under a lock: contexts on several threads may launch first together).
static cudaError_t ensure_piece_attrs() {
    static std::mutex mu;
    static bool done[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> g(mu);
    if (done[dev]) return cudaSuccess;
    e = cudaFuncSetAttribute(crc_piece_kernel<false, kCrcUnroll, kCrcThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kPieceSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(crc_piece_kernel<true, kCopyUnroll, kCopyThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kPieceSmem);
    if (e == cudaSuccess) done[dev] = true;
    return e;
}

cudaError_t launch_crc_plan(FrameJob *job, CrcTarget *targets, CrcPiece *pieces, uint32_t *crc_out,
                            uint32_t ntargets_hint, uint64_t align_base, int by_dst, int sms, cudaStream_t s) {
    const uint32_t warps = ntargets_hint ? ntargets_hint : 1;
    const uint32_t blocks = (uint32_t)std::min<uint64_t>((warps + 7) / 8, (uint64_t)sms * 8);
    crc_plan_kernel<<<blocks, 256, 0, s>>>(job, targets, pieces, crc_out, align_base, by_dst);
    return cudaGetLastError();
}

cudaError_t launch_crc_pieces(const uint8_t *src, uint8_t *dst, FrameJob *job, const CrcPiece *pieces,
                              uint32_t *crc_out, int copy, int grid, cudaStream_t s) {
    cudaError_t e = ensure_piece_attrs();
    if (e != cudaSuccess) return e;
    if (copy)
        crc_piece_kernel<true, kCopyUnroll, kCopyThreads><<<grid, kCopyThreads, kPieceSmem, s>>>(src, dst, job, pieces, crc_out);
    else
        crc_piece_kernel<false, kCrcUnroll, kCrcThreads><<<grid, kCrcThreads, kPieceSmem, s>>>(src, dst, job, pieces, crc_out);
    return cudaGetLastError();
}

cudaError_t launch_frame_heads(uint8_t *dst, const FrameJob *job, const CrcTarget *targets,
                               const uint32_t *crc_out, uint32_t n, uint64_t term_off, cudaStream_t s) {
    const uint32_t blocks = (n + 1 + 255) / 256;
    frame_heads_kernel<<<blocks, 256, 0, s>>>(dst, job, targets, crc_out, term_off);
    return cudaGetLastError();
}

cudaError_t launch_frame_walk(const uint8_t *src, uint64_t len, uint32_t max_frames, FrameJob *job,
                              CrcTarget *targets, WalkEntry *walk, WalkCand *cand, uint64_t align_base, int sms,
                              cudaStream_t s) {
    static std::mutex mu;
    static bool done[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    {
        std::lock_guard<std::mutex> g(mu);
        if (!done[dev]) {
            e = cudaFuncSetAttribute(frame_chain_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kChainSmem);
            if (e != cudaSuccess) return e;
            done[dev] = true;
        }
    }
    frame_walk_kernel<<<1, 32, 0, s>>>(src, len, max_frames, job, targets, walk);
    frame_scan_kernel<<<sms * 4, 256, 0, s>>>(src, len, job, cand);
    frame_chain_kernel<<<1, 1024, kChainSmem, s>>>(src, len, max_frames, job, targets, walk, cand);
    piece_bases_kernel<<<1, 1024, 0, s>>>(job, targets, align_base);
    return cudaGetLastError();
}

cudaError_t launch_frame_verify(const FrameJob *job, WalkEntry *walk, const uint32_t *crc_out, uint32_t max_frames,
                                cudaStream_t s) {
    const uint32_t blocks = std::max<uint32_t>(1, std::min<uint32_t>((max_frames + 255) / 256, 1024));
    frame_verify_kernel<<<blocks, 256, 0, s>>>(job, walk, crc_out);
    return cudaGetLastError();
}

cudaError_t launch_stream_locs(const uint8_t *src, const PayloadRef *payloads, uint32_t n, FrameJob *job,
                               CrcTarget *targets, int32_t *status, uint64_t align_base, cudaStream_t s) {
    const uint32_t blocks = std::max<uint32_t>(1, std::min<uint32_t>((n + 255) / 256, 1024));
    stream_locs_kernel<<<blocks, 256, 0, s>>>(src, payloads, n, job, targets, status);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    piece_bases_kernel<<<1, 1024, 0, s>>>(job, targets, align_base);
    return cudaGetLastError();
}

}  // namespace fqxv
