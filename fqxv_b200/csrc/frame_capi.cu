// C ABI of the CRC-32C and block-frame calls (include/fqxv_frame_gpu.h):
// planning on the host, one pass of frame_kernels.cu on the context's stream.
#include <algorithm>
#include <cstring>
#include <vector>

#include "frame_internal.cuh"
#include "rans_ctx.cuh"

using namespace fqxv;

namespace {

// The job header takes the first 256 bytes of the target arena, so the
// targets after it stay aligned.
constexpr size_t kJobBytes = 256;

struct Pass {
    FrameJob *job;
    CrcTarget *targets;
    CrcPiece *pieces;
    uint32_t *crc_out;
};

// Arena room for a pass of n targets and np pieces (`extra` more bytes after
// the targets, e.g. walk entries).
int ensure_pass(fqxv_rans_ctx *ctx, size_t n, uint64_t np, size_t extra, Pass *p) {
    cudaStream_t s = ctx->stream;
    CK(ctx->f_targets.ensure(kJobBytes + sizeof(CrcTarget) * std::max<size_t>(n, 1) + extra, s));
    CK(ctx->f_pieces.ensure(sizeof(CrcPiece) * std::max<uint64_t>(np, 1), s));
    CK(ctx->f_out.ensure(sizeof(uint32_t) * std::max<size_t>(n, 1), s));
    p->job = ctx->f_targets.as<FrameJob>();
    p->targets = reinterpret_cast<CrcTarget *>(ctx->f_targets.as<uint8_t>() + kJobBytes);
    p->pieces = ctx->f_pieces.as<CrcPiece>();
    p->crc_out = ctx->f_out.as<uint32_t>();
    return FQXV_RANS_OK;
}

// Upper bound of the pieces of targets whose lengths sum to `total` (any
// alignment, any piece size the device may pick).
uint64_t pieces_bound(size_t n, uint64_t total) { return (total >> kCrcMinShift) + 2 * (uint64_t)n + 1; }

// One CRC pass over targets planned on the host: the job header and targets
// go up in one copy; for a copy pass (d_dst set) the payloads are copied to
// their dst_off as they are checksummed and the frame heads written after.
// h_crcs (may be null) receives the CRCs. term_off: terminator frame offset
// in d_dst, or ~0.
int crc_pass(fqxv_rans_ctx *ctx, const uint8_t *d_src, uint8_t *d_dst, std::vector<CrcTarget> &tg,
             uint32_t *h_crcs, uint64_t term_off) {
    cudaStream_t s = ctx->stream;
    const size_t n = tg.size();
    const bool copy = d_dst != nullptr;
    uint64_t total = 0;
    for (auto &t : tg) total += t.len;
    const int psh = crc_piece_shift(total, kCrcPieceTarget, kCrcMinShift, kCrcMaxShift);
    const uint64_t align_base = reinterpret_cast<uint64_t>(copy ? (const uint8_t *)d_dst : d_src);
    uint64_t np = 0;
    for (auto &t : tg) {
        t.piece_base = np;
        np += crc_piece_count(align_base + (copy ? t.dst_off : t.src_off), t.len, psh);
    }
    if (np > 0xFFFFFFFFull || n > 0xFFFFFFFFull) return FQXV_RANS_E_TOO_LARGE;
    Pass p;
    int st = ensure_pass(ctx, n, np, 0, &p);
    if (st) return st;
    const size_t up = kJobBytes + sizeof(CrcTarget) * n;
    CK(ctx->h_stage.ensure(up + sizeof(uint32_t) * n));
    uint8_t *hs = static_cast<uint8_t *>(ctx->h_stage.p);
    FrameJob job{};
    job.ntargets = (uint32_t)n;
    job.npieces = (uint32_t)np;
    job.piece_shift = psh;
    std::memcpy(hs, &job, sizeof job);
    if (n) std::memcpy(hs + kJobBytes, tg.data(), sizeof(CrcTarget) * n);
    CK(cudaMemcpyAsync(p.job, hs, up, cudaMemcpyHostToDevice, s));
    cudaEvent_t t0 = ctx->timer.begin(s);
    CK(launch_crc_plan(p.job, p.targets, p.pieces, p.crc_out, (uint32_t)n, align_base, copy ? 1 : 0, ctx->sms,
                       s));
    ctx->timer.end(kStCrcPlan, t0, s);
    t0 = ctx->timer.begin(s);
    CK(launch_crc_pieces(d_src, d_dst, p.job, p.pieces, p.crc_out, copy ? 1 : 0, ctx->sms, s));
    ctx->timer.end(copy ? kStFrameCopy : kStCrc, t0, s);
    if (copy) CK(launch_frame_heads(d_dst, p.job, p.targets, p.crc_out, (uint32_t)n, term_off, s));
    uint32_t *hc = reinterpret_cast<uint32_t *>(hs + up);
    if (n) CK(cudaMemcpyAsync(hc, p.crc_out, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    ctx->timer.collect();
    ctx->timer.bytes[copy ? kStFrameCopy : kStCrc] += copy ? 2 * total : total;
    if (h_crcs && n) std::memcpy(h_crcs, hc, sizeof(uint32_t) * n);
    return FQXV_RANS_OK;
}

// Copies the host bytes [lo, hi) to the context's input staging; returns the
// device pointer that stands for h_src[0] (valid from lo on).
int stage_in(fqxv_rans_ctx *ctx, const uint8_t *h_src, uint64_t lo, uint64_t hi, const uint8_t **d_base) {
    cudaStream_t s = ctx->stream;
    CK(ctx->io_in.ensure(std::max<uint64_t>(hi - lo, 16), s));
    if (hi > lo) CK(cudaMemcpyAsync(ctx->io_in.p, h_src + lo, hi - lo, cudaMemcpyHostToDevice, s));
    *d_base = ctx->io_in.as<uint8_t>() - lo;
    return FQXV_RANS_OK;
}

void span_extent(const fqxv_rans_span *sp, size_t n, uint64_t *lo, uint64_t *hi) {
    uint64_t a = ~0ull, b = 0;
    for (size_t i = 0; i < n; i++) {
        if (!sp[i].length) continue;
        a = std::min<uint64_t>(a, sp[i].offset);
        b = std::max<uint64_t>(b, sp[i].offset + sp[i].length);
    }
    *lo = a == ~0ull ? 0 : a;
    *hi = b;
}

int crc_batch_impl(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *spans, size_t n,
                   uint32_t *crcs) {
    std::vector<CrcTarget> tg(n);
    for (size_t i = 0; i < n; i++) tg[i] = CrcTarget{spans[i].offset, spans[i].length, 0, 0};
    return crc_pass(ctx, d_src, nullptr, tg, crcs, ~0ull);
}

int frame_impl(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *payloads, size_t n, int terminate,
               uint8_t *d_dst, uint64_t dst_cap, uint64_t *frame_offsets, uint32_t *crcs, uint64_t *total) {
    const uint64_t need = fqxv_frame_blocks_bound(payloads, n, terminate);
    if (total) *total = need;
    if (need > dst_cap) return FQXV_RANS_E_DST_TOO_SMALL;
    std::vector<CrcTarget> tg(n);
    uint64_t pos = 0;
    for (size_t i = 0; i < n; i++) {
        tg[i] = CrcTarget{payloads[i].offset, payloads[i].length, pos + kFrameHead, 0};
        if (frame_offsets) frame_offsets[i] = pos;
        pos += kFrameHead + payloads[i].length;
    }
    return crc_pass(ctx, d_src, d_dst, tg, crcs, terminate ? pos : ~0ull);
}

int read_impl(fqxv_rans_ctx *ctx, const uint8_t *d_src, uint64_t len, size_t max_frames, fqxv_rans_span *payloads,
              uint32_t *crcs, int32_t *status, size_t *nframes, uint64_t *consumed, int *terminated) {
    cudaStream_t s = ctx->stream;
    // a frame that passes the structural checks takes at least 17 bytes, and
    // the walk stops at the first one that fails
    const uint64_t cap = std::min<uint64_t>(max_frames, len / 16 + 1);
    if (cap > 0xFFFFFFFFull) return FQXV_RANS_E_TOO_LARGE;
    Pass p;
    const size_t walk_bytes = sizeof(WalkEntry) * (size_t)std::max<uint64_t>(cap, 1);
    const size_t cand_bytes = sizeof(WalkCand) * kChainMax;
    int st = ensure_pass(ctx, (size_t)cap, pieces_bound((size_t)cap, len), walk_bytes + cand_bytes, &p);
    if (st) return st;
    WalkEntry *walk = reinterpret_cast<WalkEntry *>(p.targets + std::max<uint64_t>(cap, 1));
    WalkCand *cand = reinterpret_cast<WalkCand *>(walk + std::max<uint64_t>(cap, 1));
    const uint64_t align_base = reinterpret_cast<uint64_t>(d_src);
    cudaEvent_t t0 = ctx->timer.begin(s);
    CK(launch_frame_walk(d_src, len, (uint32_t)cap, p.job, p.targets, walk, cand, align_base, ctx->sms, s));
    ctx->timer.end(kStFrameWalk, t0, s);
    t0 = ctx->timer.begin(s);
    CK(launch_crc_plan(p.job, p.targets, p.pieces, p.crc_out, (uint32_t)cap, align_base, 0, ctx->sms, s));
    ctx->timer.end(kStCrcPlan, t0, s);
    t0 = ctx->timer.begin(s);
    CK(launch_crc_pieces(d_src, nullptr, p.job, p.pieces, p.crc_out, 0, ctx->sms, s));
    ctx->timer.end(kStCrc, t0, s);
    CK(launch_frame_verify(p.job, walk, p.crc_out, (uint32_t)cap, s));
    CK(ctx->h_stage.ensure(sizeof(FrameJob) + walk_bytes));
    uint8_t *hs = static_cast<uint8_t *>(ctx->h_stage.p);
    CK(cudaMemcpyAsync(hs, p.job, sizeof(FrameJob), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    FrameJob job;
    std::memcpy(&job, hs, sizeof job);
    WalkEntry *hw = reinterpret_cast<WalkEntry *>(hs + sizeof(FrameJob));
    if (job.nframes)
        CK(cudaMemcpyAsync(hw, walk, sizeof(WalkEntry) * job.nframes, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    ctx->timer.collect();
    uint64_t verified = 0;
    int first = FQXV_RANS_OK;
    for (uint32_t k = 0; k < job.nframes; k++) {
        const WalkEntry &e = hw[k];
        payloads[k].offset = e.pay_off;
        payloads[k].length = e.pay_len;
        if (crcs) crcs[k] = e.target == ~0u ? 0 : e.crc;
        status[k] = e.status;
        if (e.target != ~0u) verified += e.pay_len;
        if (e.status != FQXV_RANS_OK && first == FQXV_RANS_OK) first = e.status;
    }
    ctx->timer.bytes[kStCrc] += verified;
    *nframes = job.nframes;
    *consumed = job.consumed;
    *terminated = job.terminated;
    return first;
}

}  // namespace

extern "C" {

uint32_t fqxv_crc32c_combine(uint32_t crc_a, uint32_t crc_b, uint64_t len_b) {
    // crc.rs:116-161. Appending len_b zero bytes to A multiplies its CRC
    // register by x^(8 len_b) mod P; the factors x^(8 2^k) come from repeated
    // squaring (reflected representation: bit 31 holds x^0).
    if (len_b == 0) return crc_a;
    auto mul = [](uint32_t a, uint32_t b) {
        uint32_t p = 0;
        for (int i = 31; i >= 0; i--) {
            if ((a >> i) & 1u) p ^= b;
            b = (b >> 1) ^ ((b & 1u) ? 0x82F63B78u : 0u);
        }
        return p;
    };
    uint32_t sq = 0x80000000u >> 8;  // x^8
    uint32_t f = 0x80000000u;        // 1
    for (uint64_t n = len_b; n; n >>= 1) {
        if (n & 1) f = mul(f, sq);
        sq = mul(sq, sq);
    }
    return mul(crc_a, f) ^ crc_b;
}

uint64_t fqxv_frame_blocks_bound(const fqxv_rans_span *payloads, size_t n, int terminate) {
    uint64_t t = terminate ? kFrameTerm : 0;
    for (size_t i = 0; i < n; i++) t += kFrameHead + payloads[i].length;
    return t;
}

int fqxv_crc32c_batch(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *spans, size_t n,
                      uint32_t *crcs) {
    if (!ctx || (n && (!spans || !crcs || !d_src))) return FQXV_RANS_E_INVALID_ARG;
    std::lock_guard<std::mutex> g(ctx->mu);
    DeviceGuard dg(ctx->device);
    return crc_batch_impl(ctx, d_src, spans, n, crcs);
}

int fqxv_crc32c_batch_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, const fqxv_rans_span *spans, size_t n,
                           uint32_t *crcs) {
    if (!ctx || (n && (!spans || !crcs || !h_src))) return FQXV_RANS_E_INVALID_ARG;
    std::lock_guard<std::mutex> g(ctx->mu);
    DeviceGuard dg(ctx->device);
    uint64_t lo, hi;
    span_extent(spans, n, &lo, &hi);
    const uint8_t *d_base = nullptr;
    int st = stage_in(ctx, h_src, lo, hi, &d_base);
    if (st) return st;
    return crc_batch_impl(ctx, d_base, spans, n, crcs);
}

int fqxv_frame_blocks(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *payloads, size_t n,
                      int terminate, uint8_t *d_dst, uint64_t dst_cap, uint64_t *frame_offsets, uint32_t *crcs,
                      uint64_t *total) {
    if (!ctx || !d_dst || (n && (!payloads || !d_src))) return FQXV_RANS_E_INVALID_ARG;
    std::lock_guard<std::mutex> g(ctx->mu);
    DeviceGuard dg(ctx->device);
    return frame_impl(ctx, d_src, payloads, n, terminate, d_dst, dst_cap, frame_offsets, crcs, total);
}

int fqxv_frame_blocks_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, const fqxv_rans_span *payloads, size_t n,
                           int terminate, uint8_t *h_dst, uint64_t dst_cap, uint64_t *frame_offsets,
                           uint32_t *crcs, uint64_t *total) {
    if (!ctx || !h_dst || (n && (!payloads || !h_src))) return FQXV_RANS_E_INVALID_ARG;
    std::lock_guard<std::mutex> g(ctx->mu);
    DeviceGuard dg(ctx->device);
    const uint64_t need = fqxv_frame_blocks_bound(payloads, n, terminate);
    if (total) *total = need;
    if (need > dst_cap) return FQXV_RANS_E_DST_TOO_SMALL;
    uint64_t lo, hi;
    span_extent(payloads, n, &lo, &hi);
    const uint8_t *d_base = nullptr;
    int st = stage_in(ctx, h_src, lo, hi, &d_base);
    if (st) return st;
    cudaStream_t s = ctx->stream;
    CK(ctx->io_out.ensure(std::max<uint64_t>(need, 16), s));
    st = frame_impl(ctx, d_base, payloads, n, terminate, ctx->io_out.as<uint8_t>(), need, frame_offsets, crcs,
                    nullptr);
    if (st) return st;
    if (need) CK(cudaMemcpyAsync(h_dst, ctx->io_out.p, need, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return FQXV_RANS_OK;
}

int fqxv_read_blocks(fqxv_rans_ctx *ctx, const uint8_t *d_src, uint64_t len, size_t max_frames,
                     fqxv_rans_span *payloads, uint32_t *crcs, int32_t *status, size_t *nframes, uint64_t *consumed,
                     int *terminated) {
    if (!ctx || !nframes || !consumed || !terminated || (max_frames && (!payloads || !status)) ||
        (len && !d_src))
        return FQXV_RANS_E_INVALID_ARG;
    std::lock_guard<std::mutex> g(ctx->mu);
    DeviceGuard dg(ctx->device);
    return read_impl(ctx, d_src, len, max_frames, payloads, crcs, status, nframes, consumed, terminated);
}

int fqxv_read_blocks_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, uint64_t len, size_t max_frames,
                          fqxv_rans_span *payloads, uint32_t *crcs, int32_t *status, size_t *nframes,
                          uint64_t *consumed, int *terminated) {
    if (!ctx || !nframes || !consumed || !terminated || (max_frames && (!payloads || !status)) ||
        (len && !h_src))
        return FQXV_RANS_E_INVALID_ARG;
    std::lock_guard<std::mutex> g(ctx->mu);
    DeviceGuard dg(ctx->device);
    const uint8_t *d_base = nullptr;
    int st = stage_in(ctx, h_src, 0, len, &d_base);
    if (st) return st;
    return read_impl(ctx, d_base, len, max_frames, payloads, crcs, status, nframes, consumed, terminated);
}

int fqxv_payload_stream_locs(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *payloads, size_t n,
                             uint64_t base, fqxv_stream_loc *locs, int32_t *status) {
    if (!ctx || (n && (!payloads || !locs || !status || !d_src))) return FQXV_RANS_E_INVALID_ARG;
    if (n == 0) return FQXV_RANS_OK;
    if (3 * (uint64_t)n > 0xFFFFFFFFull) return FQXV_RANS_E_TOO_LARGE;
    std::lock_guard<std::mutex> g(ctx->mu);
    DeviceGuard dg(ctx->device);
    cudaStream_t s = ctx->stream;
    uint64_t total = 0;
    for (size_t i = 0; i < n; i++) total += payloads[i].length;
    const size_t nt = 3 * n;
    const size_t ref_bytes = sizeof(PayloadRef) * n;
    const size_t st_bytes = sizeof(int32_t) * n;
    Pass p;
    int st = ensure_pass(ctx, nt, pieces_bound(nt, total), ref_bytes + st_bytes, &p);
    if (st) return st;
    PayloadRef *d_refs = reinterpret_cast<PayloadRef *>(p.targets + nt);
    int32_t *d_status = reinterpret_cast<int32_t *>(d_refs + n);
    CK(ctx->h_stage.ensure(ref_bytes + sizeof(CrcTarget) * nt + sizeof(uint32_t) * nt + st_bytes));
    uint8_t *hs = static_cast<uint8_t *>(ctx->h_stage.p);
    PayloadRef *hr = reinterpret_cast<PayloadRef *>(hs);
    for (size_t i = 0; i < n; i++) hr[i] = PayloadRef{payloads[i].offset, payloads[i].length};
    CK(cudaMemcpyAsync(d_refs, hr, ref_bytes, cudaMemcpyHostToDevice, s));
    const uint64_t align_base = reinterpret_cast<uint64_t>(d_src);
    CK(launch_stream_locs(d_src, d_refs, (uint32_t)n, p.job, p.targets, d_status, align_base, s));
    cudaEvent_t t0 = ctx->timer.begin(s);
    CK(launch_crc_plan(p.job, p.targets, p.pieces, p.crc_out, (uint32_t)nt, align_base, 0, ctx->sms, s));
    ctx->timer.end(kStCrcPlan, t0, s);
    t0 = ctx->timer.begin(s);
    CK(launch_crc_pieces(d_src, nullptr, p.job, p.pieces, p.crc_out, 0, ctx->sms, s));
    ctx->timer.end(kStCrc, t0, s);
    CrcTarget *ht = reinterpret_cast<CrcTarget *>(hs + ref_bytes);
    uint32_t *hc = reinterpret_cast<uint32_t *>(ht + nt);
    int32_t *hst = reinterpret_cast<int32_t *>(hc + nt);
    CK(cudaMemcpyAsync(ht, p.targets, sizeof(CrcTarget) * nt, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hc, p.crc_out, sizeof(uint32_t) * nt, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hst, d_status, st_bytes, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    ctx->timer.collect();
    int first = FQXV_RANS_OK;
    for (size_t i = 0; i < n; i++) {
        status[i] = hst[i];
        for (int k = 0; k < 3; k++) {
            const CrcTarget &t = ht[3 * i + k];
            fqxv_stream_loc &l = locs[3 * i + k];
            if (hst[i] == FQXV_RANS_OK) {
                l.offset = base + t.src_off;
                l.len = (uint32_t)t.len;
                l.crc = hc[3 * i + k];
                ctx->timer.bytes[kStCrc] += t.len;
            } else {
                l.offset = 0;
                l.len = 0;
                l.crc = 0;
            }
        }
        if (hst[i] != FQXV_RANS_OK && first == FQXV_RANS_OK) first = hst[i];
    }
    return first;
}

}  // extern "C"
