// C ABI of libfqxv_rans_gpu.so: contexts, device arenas, the batched device
// API and the reference-shaped single-call host API (include/fqxv_rans_gpu.h).
#include <algorithm>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numeric>
#include <thread>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/fqxv_streams_gpu.h"
#include "../../include/fqxv_rans_gpu_testing.h"
#include "../../include/fqxv_rans_x_gpu.h"
#include "../../include/fqxv_tok_gpu.h"
#include "frame_internal.cuh"
#include "rans_ctx.cuh"

using namespace fqxv;

namespace fqxv {
int sm_count(int device) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 148;
    return v > 0 ? v : 148;
}
}  // namespace fqxv

namespace {

uint64_t enc_bound_one(uint64_t n, int order) {
    if (n == 0) return kHdr;
    const uint64_t tables = order == FQXV_RANS_ORDER0 ? kO0Tables : kO1Bitmap + 256 * kO1Table;
    return kHdr + tables + kStatesBytes + 2 * n;
}

// Smallest batch output mirrored into a pinned host destination by the
// decoding CTAs, and fewest streams whose pinned input is read in place.
constexpr uint64_t kZeroCopyMinBytes = 4ull << 20;
constexpr size_t kZeroCopyMinStreams = 256;

}  // namespace

// Device address of a pinned, mapped host buffer (nullptr for any other
// memory).
void *fqxv::mapped_device_ptr(const void *h) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, h) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (a.type != cudaMemoryTypeHost) return nullptr;
    return a.devicePointer;
}

namespace {

// NVTX range for the lifetime of a scope: the batch calls and their stages
// show up by name in a timeline profiler (no cost without one attached).
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};

int encode_batch_impl(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *blocks,
                      size_t nb, int mode, uint8_t *d_dst, uint64_t dst_cap, fqxv_rans_span *out_spans,
                      int32_t *out_orders, int persistent) {
    if (mode < FQXV_RANS_ORDER0 || mode > FQXV_RANS_BEST_TIE1) return FQXV_RANS_E_INVALID_ARG;
    if (nb == 0) return FQXV_RANS_OK;
    if (nb > (1u << 30)) return FQXV_RANS_E_TOO_LARGE;
    NvtxRange range("fqxv.encode_batch");
    cudaStream_t s = ctx->stream;
    const bool o0 = mode != FQXV_RANS_ORDER1, o1 = mode != FQXV_RANS_ORDER0;

    std::vector<EncBlock> hb(nb);
    uint64_t woff = 0, toff = 0, bound = 0;
    for (size_t i = 0; i < nb; i++) {
        EncBlock &B = hb[i];
        std::memset(&B, 0, sizeof B);
        B.src_off = blocks[i].offset;
        B.n = blocks[i].length;
        B.mode = mode;
        B.word_off[0] = woff;
        if (o0) woff += B.n;
        B.word_off[1] = woff;
        if (o1) woff += B.n;
        B.tbl_off = toff;
        toff += align_up(o1 ? enc_table_bytes(B.n) : kTblUmap, 256);
        bound += enc_bound_one(B.n, o1 ? FQXV_RANS_ORDER1 : FQXV_RANS_ORDER0);
    }
    // Largest blocks first: the model kernel strides over this order and the
    // encode queue hands jobs out in it (longest-processing-time first).
    std::vector<uint32_t> ord(nb);
    std::iota(ord.begin(), ord.end(), 0u);
    std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) { return hb[a].n > hb[b].n; });
    std::vector<EncJob> jobs;
    jobs.reserve(nb * 2);
    for (uint32_t b : ord) {
        if (o1) jobs.push_back({b, 1});
        if (o0) jobs.push_back({b, 0});
    }
    // The model kernel: blocks of kModelClusterMin bytes or more get a
    // cluster of kModelCluster CTAs each, smaller ones one CTA each (a
    // cluster's barriers would cost more than their histogram); as many
    // clusters as are resident at once.
    size_t nlarge = 0;
    while (nlarge < nb && hb[ord[nlarge]].n >= kModelClusterMin) nlarge++;
    const int grid_large = (int)std::min<size_t>(nlarge, std::max<size_t>(1, (size_t)ctx->sms * 4 / kModelCluster));
    const int grid_small = (int)std::min<size_t>(nb - nlarge, (size_t)ctx->sms * 2);
    const int model_grid = std::max(grid_large, grid_small);
    CK(ctx->e_blocks.ensure(nb * sizeof(EncBlock), s));
    CK(ctx->e_order.ensure(nb * sizeof(uint32_t), s));
    CK(ctx->e_jobs.ensure(jobs.size() * sizeof(EncJob), s));
    CK(ctx->e_tbl.ensure(std::max<uint64_t>(toff, 256), s));
    CK(ctx->e_words.ensure(std::max<uint64_t>(woff * 2, 16), s));
    CK(ctx->e_hist.ensure(o1 ? (size_t)model_grid * 65536 * 4 : 256, s));
    // order-1: each input position's table index (u16), written by the
    // model and read by the encode
    uint64_t src_end = 0;
    for (size_t i = 0; i < nb; i++) src_end = std::max<uint64_t>(src_end, blocks[i].offset + blocks[i].length);
    const bool keyed = o1 && ctx->tune.enc_o1_keys;
    if (keyed) CK(ctx->e_keys.ensure(2 * (src_end + 16), s));
    uint16_t *dK = keyed ? ctx->e_keys.as<uint16_t>() : nullptr;
    CK(ctx->e_misc.ensure((2 + nb) * 16, s));
    // Stage descriptors through pinned memory, one copy per array.
    const size_t szb = nb * sizeof(EncBlock), szo = nb * 4, szj = jobs.size() * sizeof(EncJob);
    CK(ctx->h_stage.ensure(szb + szo + szj + 64));
    cudaStreamSynchronize(s);  // the staging buffer may still feed an earlier copy
    uint8_t *hs = (uint8_t *)ctx->h_stage.p;
    std::memcpy(hs, hb.data(), szb);
    std::memcpy(hs + szb, ord.data(), szo);
    std::memcpy(hs + szb + szo, jobs.data(), szj);
    CK(cudaMemcpyAsync(ctx->e_blocks.p, hs, szb, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->e_order.p, hs + szb, szo, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->e_jobs.p, hs + szb + szo, szj, cudaMemcpyHostToDevice, s));
    int *queue = ctx->e_misc.as<int>();
    uint64_t *total = reinterpret_cast<uint64_t *>(ctx->e_misc.as<uint8_t>() + 16);
    CK(cudaMemsetAsync(queue, 0, 16, s));

    EncBlock *dB = ctx->e_blocks.as<EncBlock>();
    const uint32_t *dO = ctx->e_order.as<uint32_t>();
    const EncJob *dJ = ctx->e_jobs.as<EncJob>();
    uint8_t *dT = ctx->e_tbl.as<uint8_t>();
    uint16_t *dW = ctx->e_words.as<uint16_t>();
    uint32_t *dH = ctx->e_hist.as<uint32_t>();
    // A batch whose largest block is far above its mean has a serial tail:
    // its largest jobs run faster with fewer warps per scheduler
    // (enc_run_ctas_per_sm). A batch of like-sized blocks is throughput-bound
    // and takes enc_run_ctas_per_sm_uniform.
    uint64_t nsum = 0, nmax = 0;
    for (size_t i = 0; i < nb; i++) {
        nsum += hb[i].n;
        nmax = std::max<uint64_t>(nmax, hb[i].n);
    }
    const bool tail = (double)nmax > 4.0 * (double)nsum / (double)nb;
    const int run_grid = ctx->sms * (int)(tail ? ctx->tune.enc_run_ctas_per_sm : ctx->tune.enc_run_ctas_per_sm_uniform);
    if (persistent) {
        cudaEvent_t t0;
        if (nlarge) {
            t0 = ctx->timer.begin(s);
            CK(launch_enc_model(d_src, dB, dO, (int)nlarge, dT, dH, dK, grid_large, kModelCluster, s));
            ctx->timer.end(kStEncModel, t0, s);
        }
        if (nb > nlarge) {
            t0 = ctx->timer.begin(s);
            CK(launch_enc_model(d_src, dB, dO + nlarge, (int)(nb - nlarge), dT, dH, dK, grid_small, 1, s));
            ctx->timer.end(kStEncModel, t0, s);
        }
        t0 = ctx->timer.begin(s);
        launch_enc_run(d_src, dB, dJ, (int)jobs.size(), dT, dW, queue, dK,
                       std::min<int>(run_grid, (int)(jobs.size() + 3) / 4), s);
        ctx->timer.end(kStEncRun, t0, s);
    } else {
        // The plain form: every block gets its own launches, one after the other.
        const int per = (o0 && o1) ? 2 : 1;
        for (size_t j = 0; j < nb; j++) {
            CK(cudaMemsetAsync(queue, 0, 4, s));
            cudaEvent_t t0 = ctx->timer.begin(s);
            CK(launch_enc_model(d_src, dB, dO + j, 1, dT, dH, dK, 1, kModelCluster, s));
            ctx->timer.end(kStEncModel, t0, s);
            t0 = ctx->timer.begin(s);
            launch_enc_run(d_src, dB, dJ + j * per, per, dT, dW, queue, dK, 1, s);
            ctx->timer.end(kStEncRun, t0, s);
        }
    }
    {
        cudaEvent_t t0 = ctx->timer.begin(s);
        launch_enc_select_scan(dB, (int)nb, total, s);
        ctx->timer.end(kStEncScan, t0, s);
    }
    CK(cudaGetLastError());
    if (bound > dst_cap) {
        uint64_t tot = 0;
        CK(cudaMemcpyAsync(&tot, total, 8, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (tot > dst_cap) return FQXV_RANS_E_DST_TOO_SMALL;
    }
    if (persistent) {
        cudaEvent_t t0 = ctx->timer.begin(s);
        launch_enc_pack(dB, (int)nb, dT, dW, d_dst, (int)std::min<size_t>(nb * kPackParts, (size_t)ctx->sms * 8),
                        s);
        ctx->timer.end(kStEncPack, t0, s);
    } else {
        for (size_t j = 0; j < nb; j++) {
            cudaEvent_t t0 = ctx->timer.begin(s);
            launch_enc_pack(dB + j, 1, dT, dW, d_dst, kPackParts, s);
            ctx->timer.end(kStEncPack, t0, s);
        }
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(hs, dB, szb, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    ctx->timer.collect();
    const EncBlock *rb = reinterpret_cast<const EncBlock *>(hs);
    for (size_t i = 0; i < nb; i++) {
        // Algorithmic bytes per stage: the model reads the block, each encode
        // job reads it and writes its words, the pack reads the chosen words
        // and writes the stream.
        ctx->timer.bytes[kStEncModel] += rb[i].n;
        if (o0) ctx->timer.bytes[kStEncRun] += rb[i].n + 2 * rb[i].nwords[0];
        if (o1) ctx->timer.bytes[kStEncRun] += rb[i].n + 2 * rb[i].nwords[1];
        ctx->timer.bytes[kStEncPack] += 2 * rb[i].nwords[rb[i].chosen] + rb[i].out_size[rb[i].chosen];
    }
    for (size_t i = 0; i < nb; i++) {
        out_spans[i].offset = rb[i].out_off;
        out_spans[i].length = rb[i].out_size[rb[i].chosen];
        if (out_orders) out_orders[i] = rb[i].chosen;
    }
    return FQXV_RANS_OK;
}

int decode_batch_impl(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *blocks, size_t nb,
                      uint64_t max_len, uint8_t *d_dst, const fqxv_rans_span *out_spans, uint64_t *out_lens,
                      int32_t *status, int persistent, uint8_t *mirror = nullptr) {
    if (nb == 0) return FQXV_RANS_OK;
    if (nb > (1u << 30)) return FQXV_RANS_E_TOO_LARGE;
    NvtxRange range("fqxv.decode_batch");
    cudaStream_t s = ctx->stream;
    std::vector<DecStream> hs(nb);
    uint64_t toff = 0;
    for (size_t i = 0; i < nb; i++) {
        DecStream &S = hs[i];
        std::memset(&S, 0, sizeof S);
        S.src_off = blocks[i].offset;
        S.src_len = blocks[i].length;
        S.dst_off = out_spans[i].offset;
        S.dst_cap = out_spans[i].length;
        S.max_len = max_len;
        S.tbl_off = toff;
        toff += align_up(dec_table_bytes(S.src_len), 256);
    }
    std::vector<uint32_t> ord(nb);
    std::iota(ord.begin(), ord.end(), 0u);
    std::stable_sort(ord.begin(), ord.end(),
                     [&](uint32_t a, uint32_t b) { return hs[a].dst_cap > hs[b].dst_cap; });
    CK(ctx->d_streams.ensure(nb * sizeof(DecStream), s));
    CK(ctx->d_order.ensure(nb * 4, s));
    CK(ctx->d_tbl.ensure(std::max<uint64_t>(toff, 256), s));
    CK(ctx->d_misc.ensure(512, s));
    const size_t szs = nb * sizeof(DecStream), szo = nb * 4;
    CK(ctx->h_stage.ensure(szs + szo + 64));
    cudaStreamSynchronize(s);
    uint8_t *hst = (uint8_t *)ctx->h_stage.p;
    std::memcpy(hst, hs.data(), szs);
    std::memcpy(hst + szs, ord.data(), szo);
    CK(cudaMemcpyAsync(ctx->d_streams.p, hst, szs, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->d_order.p, hst + szs, szo, cudaMemcpyHostToDevice, s));
    int *queue = ctx->d_misc.as<int>();
    CK(cudaMemsetAsync(queue, 0, 16, s));
    DecStream *dS = ctx->d_streams.as<DecStream>();
    uint8_t *dT = ctx->d_tbl.as<uint8_t>();
    if (persistent) {
        cudaEvent_t t0 = ctx->timer.begin(s);
        launch_dec_parse(d_src, dS, (int)nb, dT, (int)std::min<size_t>(nb, (size_t)ctx->sms * 8), s);
        ctx->timer.end(kStDecParse, t0, s);
    } else {
        for (size_t j = 0; j < nb; j++) {
            cudaEvent_t t0 = ctx->timer.begin(s);
            launch_dec_parse(d_src, dS + ord[j], 1, dT, 1, s);
            ctx->timer.end(kStDecParse, t0, s);
        }
    }
    CK(cudaGetLastError());
    // The parse decides each stream's class (order-0, order-1 with shared-
    // memory tables, order-1 with global tables); one kernel per class.
    CK(cudaMemcpyAsync(hst, dS, szs, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    {
        // Launch groups: order-0; order-1 small alphabets (one warp per
        // stream, many per SM); order-1 byte columns by table size (the
        // shared memory of a group is its largest member's); the order-1
        // streams that bound the batch by their serial time in two groups of
        // their own (below); order-1 global.
        const DecStream *ps = reinterpret_cast<const DecStream *>(hst);
        const int64_t top_max = ctx->tune.o1_top_max < 0 ? ctx->sms / 2 : ctx->tune.o1_top_max;
        // A stream whose serial decode (its rounds one after another) takes
        // longer than o1_top_latency_pct % of the whole batch's throughput-
        // bound time would finish last however the rest is packed: the
        // o1_top_max longest such order-1 streams (by serial time) form the
        // top groups -- wide alphabets on the four-warp decoder, small ones
        // on the one-warp decoder. Costs in SM cycles per byte, from B200
        // measurements: a stream's serial time is cycles per 32-byte round /
        // 32 per byte; the batch's throughput time is the sum over streams
        // of bytes x (SM cycles per byte at the class's full-GPU rate) / SMs.
        auto lat_cpb = [](const DecStream &d) {
            return d.cls == kClsO0 ? 5.0 : d.nd <= kShflMaxNd ? 15.0 : d.nd <= kSmallMaxNd ? 18.0 : 19.5;
        };
        auto rate_cpb = [](const DecStream &d) {
            return d.cls == kClsO0 ? 0.9 : d.cls == kClsO1Global ? 14.0 : d.nd <= kSmallMaxNd ? 3.0 : 7.0;
        };
        double bulk = 0;
        for (size_t i = 0; i < nb; i++)
            if (ps[i].cls != kClsNone) bulk += (double)ps[i].n * rate_cpb(ps[i]);
        const double top_thr = bulk / ctx->sms * (double)ctx->tune.o1_top_latency_pct / 100.0;
        std::vector<std::pair<double, uint32_t>> cand;
        for (size_t i = 0; i < nb; i++) {
            const DecStream &d = ps[i];
            const double lat = (double)d.n * lat_cpb(d);
            if (d.cls == kClsO1Dense && lat > top_thr) cand.emplace_back(lat, (uint32_t)i);
        }
        const size_t ntop = std::min<size_t>(cand.size(), (size_t)std::max<int64_t>(top_max, 0));
        std::partial_sort(cand.begin(), cand.begin() + ntop, cand.end(),
                          [](const std::pair<double, uint32_t> &a, const std::pair<double, uint32_t> &b) {
                              return a.first > b.first || (a.first == b.first && a.second < b.second);
                          });
        std::vector<uint8_t> is_top(nb, 0);
        for (size_t k = 0; k < ntop; k++) is_top[cand[k].second] = 1;
        auto group_of = [&](uint32_t i) -> int {
            const DecStream &d = ps[i];
            if (d.cls == kClsO0) return 0;
            if (d.cls == kClsO1Global) return kGroups - 1;
            if (d.cls != kClsO1Dense) return -1;
            if (d.nd <= kSmallMaxNd) return is_top[i] ? kGroupSmallTop : 1;
            if (is_top[i]) return kGroupFourTop;
            return d.tbl_bytes <= (uint64_t)ctx->tune.dense_edge_small   ? kGroupDense0
                   : d.tbl_bytes <= (uint64_t)ctx->tune.dense_edge_large ? kGroupDense0 + 1
                                                                         : kGroupDense0 + 2;
        };
        std::vector<uint32_t> lists[kGroups];
        uint32_t tmax[kGroups] = {}, tmaxp[kGroups] = {};
        uint64_t cbytes[kGroups] = {};
        uint64_t maxn[kGroups] = {};
        int ndmax[kGroups] = {};
        for (uint32_t i : ord) {
            const int g = group_of(i);
            if (g < 0) continue;
            lists[g].push_back(i);
            tmax[g] = std::max(tmax[g], ps[i].tbl_bytes);
            tmaxp[g] = std::max(tmaxp[g], ps[i].tbl_bytes_planes);
            cbytes[g] += ps[i].src_len + ps[i].n;
            maxn[g] = std::max<uint64_t>(maxn[g], ps[i].n);
            ndmax[g] = std::max(ndmax[g], ps[i].nd);
        }
        int gcls[kGroups];
        uint32_t smem[kGroups];
        const int64_t four_max = ctx->tune.o1_four_max_streams < 0 ? ctx->sms : ctx->tune.o1_four_max_streams;
        for (int g = 0; g < kGroups; g++) {
            if (g == 0) gcls[g] = kClsO0;
            else if (g == kGroups - 1) gcls[g] = kClsO1Global;
            else if (g == 1 || g == kGroupSmallTop) gcls[g] = kClsO1Small;
            else if (g == kGroupFourTop) gcls[g] = kClsO1Dense;
            else gcls[g] = (int64_t)lists[g].size() < four_max ? kClsO1Dense : kClsO1Wide;
            // the four-warp decoder also stages the bit-plane columns
            smem[g] = dec_smem_bytes(gcls[g], gcls[g] == kClsO1Dense ? tmaxp[g] : tmax[g], ndmax[g]);
            // the groups of largest streams: one CTA per SM, alone on it
            if ((g == kGroupFourTop || g == kGroupSmallTop) && ctx->tune.o1_top_exclusive)
                smem[g] = std::max(smem[g], dec_exclusive_smem(gcls[g], g == kGroupSmallTop
                                                                              ? (int)ctx->tune.o1_top_small_per_sm
                                                                              : 1));
        }
        // Groups are launched longest first -- by the serial time of their
        // largest stream (rounds x cycles per round: ~620 for order-1,
        // ~160 for order-0) -- so the streams that bound the batch take SMs
        // before the groups that finish early.
        int glaunch[kGroups];
        for (int g = 0; g < kGroups; g++) glaunch[g] = g;
        auto gcost = [&](int g) { return (double)maxn[g] * (g == 0 ? 160.0 : 620.0); };
        std::stable_sort(glaunch, glaunch + kGroups, [&](int a, int b) { return gcost(a) > gcost(b); });
        size_t tot = 0;
        for (int g = 0; g < kGroups; g++) tot += lists[g].size();
        CK(ctx->d_order.ensure(std::max<size_t>(tot, 1) * 4, s));
        uint32_t *hl = reinterpret_cast<uint32_t *>(hst + szs);
        size_t at = 0, base[kGroups];
        for (int g = 0; g < kGroups; g++) {
            base[g] = at;
            std::memcpy(hl + at, lists[g].data(), lists[g].size() * 4);
            at += lists[g].size();
        }
        if (tot) CK(cudaMemcpyAsync(ctx->d_order.p, hl, tot * 4, cudaMemcpyHostToDevice, s));
        CK(cudaMemsetAsync(queue, 0, 4 * 4 * kGroups, s));
        CK(cudaEventRecord(ctx->ev_fork, s));
        const uint32_t *dl = ctx->d_order.as<uint32_t>();
        for (int gi = 0; gi < kGroups; gi++) {
            const int g = glaunch[gi];
            const size_t m = lists[g].size();
            if (!m) continue;
            const int cls = gcls[g];
            const int stage = cls == kClsO0 ? kStDecO0 : cls == kClsO1Global ? kStDecO1Global
                              : cls == kClsO1Small ? kStDecO1Small : cls == kClsO1Wide ? kStDecO1Wide
                                                                                         : kStDecO1Dense;
            cudaStream_t as = ctx->aux[g];
            CK(cudaStreamWaitEvent(as, ctx->ev_fork, 0));
            int per_sm = dec_blocks_per_sm(cls, smem[g]);
            const Tuning &T = ctx->tune;
            int64_t cap = cls == kClsO0 ? T.cta_cap_o0 : cls == kClsO1Small ? T.cta_cap_o1_small
                          : cls == kClsO1Wide ? T.cta_cap_o1_wide : cls == kClsO1Dense ? T.cta_cap_o1_four
                                                                                      : T.cta_cap_o1_global;
            // A batch bound by its top groups only needs the rest done by
            // then: fewer one-warp CTAs per SM slow its largest streams less.
            if (ntop && g != kGroupSmallTop && g != kGroupFourTop) {
                if (cls == kClsO1Small) cap = std::min<int64_t>(cap, T.cta_cap_o1_small_topped);
                if (cls == kClsO1Wide) cap = std::min<int64_t>(cap, T.cta_cap_o1_wide_topped);
            }
            per_sm = std::max(1, std::min<int>(per_sm, (int)cap));
            ctx->timer.shape(stage, per_sm, smem[g]);
            if (persistent) {
                const int grid = (int)std::min<size_t>(m, (size_t)ctx->sms * per_sm);
                cudaEvent_t t0 = ctx->timer.begin(as);
                launch_dec_run(cls, d_src, dS, dl + base[g], (int)m, dT, d_dst, queue + 4 * g, grid, smem[g],
                               ctx->first_polls, mirror, as);
                ctx->timer.end(stage, t0, as);
            } else {
                for (size_t j = 0; j < m; j++) {
                    CK(cudaMemsetAsync(queue + 4 * g, 0, 4, as));
                    cudaEvent_t t0 = ctx->timer.begin(as);
                    launch_dec_run(cls, d_src, dS, dl + base[g] + j, 1, dT, d_dst, queue + 4 * g, 1,
                                   dec_smem_bytes(cls, cls == kClsO1Dense ? ps[lists[g][j]].tbl_bytes_planes
                                                                          : ps[lists[g][j]].tbl_bytes,
                                                  ps[lists[g][j]].nd),
                                   ctx->first_polls, mirror, as);
                    ctx->timer.end(stage, t0, as);
                }
            }
            ctx->timer.bytes[stage] += cbytes[g];
            CK(cudaEventRecord(ctx->ev_join[g], as));
            CK(cudaStreamWaitEvent(s, ctx->ev_join[g], 0));
        }
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(hst, dS, szs, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    ctx->timer.collect();
    const DecStream *rs = reinterpret_cast<const DecStream *>(hst);
    int first = FQXV_RANS_OK;
    for (size_t i = 0; i < nb; i++) {
        if (status) status[i] = rs[i].status;
        if (out_lens) out_lens[i] = rs[i].status == FQXV_RANS_OK ? rs[i].n : 0;
        if (rs[i].status != FQXV_RANS_OK && first == FQXV_RANS_OK) first = rs[i].status;
    }
    return first;
}

// One default context per device for the single-call API.
std::mutex g_default_mu;
fqxv_rans_ctx *g_default[64];

int default_ctx(fqxv_rans_ctx **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return FQXV_RANS_E_NO_DEVICE;
    }
    if (dev < 0 || dev >= 64) return FQXV_RANS_E_NO_DEVICE;
    std::lock_guard<std::mutex> g(g_default_mu);
    if (!g_default[dev]) {
        const int st = fqxv_rans_ctx_create(dev, &g_default[dev]);
        if (st != FQXV_RANS_OK) return st;
    }
    *out = g_default[dev];
    return FQXV_RANS_OK;
}

}  // namespace

// The batch coder for callers inside the library that already hold the
// context's lock and device (rans_ctx.cuh).
int fqxv::encode_batch_locked(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *blocks, size_t nb,
                              int mode, uint8_t *d_dst, uint64_t dst_cap, fqxv_rans_span *out_spans,
                              int32_t *out_orders) {
    return encode_batch_impl(ctx, d_src, blocks, nb, mode, d_dst, dst_cap, out_spans, out_orders, 1);
}

int fqxv::decode_batch_locked(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *blocks, size_t nb,
                              uint64_t max_len, uint8_t *d_dst, const fqxv_rans_span *out_spans,
                              uint64_t *out_lens, int32_t *status) {
    return decode_batch_impl(ctx, d_src, blocks, nb, max_len, d_dst, out_spans, out_lens, status, 1);
}

extern "C" {

const char *fqxv_rans_status_message(int status) {
    switch (status) {
        case FQXV_RANS_OK: return "ok";
        case FQXV_RANS_E_TRUNCATED: return "truncated stream";
        case FQXV_RANS_E_UNKNOWN_ORDER: return "unknown order tag";
        case FQXV_RANS_E_FREQ_EXCEEDS: return "rANS freq table exceeds TOTFREQ";
        case FQXV_RANS_E_FREQ_SUM: return "rANS freq table does not sum to TOTFREQ";
        case FQXV_RANS_E_ABSENT_CONTEXT: return "symbol references absent context";
        case FQXV_RANS_E_ALLOC: return "rANS output length too large to allocate";
        case FQXV_RANS_E_BOUND: return "rANS output length exceeds caller bound";
        case FQXV_RANS_E_TRUNCATED_RENORM: return "truncated renorm stream";
        case FQXV_RANS_E_X_MALFORMED: return "malformed extended stream";
        case FQXV_RANS_E_INVALID_ARG: return "invalid argument";
        case FQXV_RANS_E_DST_TOO_SMALL: return "destination buffer too small";
        case FQXV_RANS_E_CUDA: return "CUDA error";
        case FQXV_RANS_E_NO_DEVICE: return "no CUDA device";
        case FQXV_RANS_E_OUT_OF_MEMORY: return "device out of memory";
        case FQXV_RANS_E_TIMEOUT: return "device wait timed out";
        case FQXV_RANS_E_TOO_LARGE: return "request too large";
        // crates/fqxv/src/lib.rs:167-178 (the block index is the caller's)
        case FQXV_FRAME_E_TRUNCATED: return "truncated fqxv stream";
        case FQXV_FRAME_E_CORRUPT: return "corrupted fqxv data: block (crc mismatch)";
        case FQXV_FRAME_E_BAD_SYNC: return "corrupted fqxv data: block (bad sync marker) (crc mismatch)";
        case FQXV_FRAME_E_TOO_LARGE: return "malformed fqxv block: block payload length exceeds the maximum";
        // crates/fqxv-tokenizer/src/lib.rs Error::Malformed texts
        case FQXV_TOK_E_VERSION: return "malformed name stream: unsupported version";
        case FQXV_TOK_E_TRUNCATED: return "malformed name stream: truncated";
        case FQXV_TOK_E_VARINT: return "malformed name stream: varint too long";
        case FQXV_TOK_E_RECORDS: return "malformed name stream: record count exceeds token stream";
        case FQXV_TOK_E_SYM_UNDERRUN: return "malformed name stream: op sym underrun";
        case FQXV_TOK_E_RUN_TOO_LONG: return "malformed name stream: op run too long";
        case FQXV_TOK_E_OPS_BOUND: return "malformed name stream: op columns exceed the stream bound";
        case FQXV_TOK_E_PLANE_LEN: return "malformed name stream: delta plane length mismatch";
        case FQXV_TOK_E_MATCH: return "malformed name stream: MATCH without prior token";
        case FQXV_TOK_E_STR_UNDERRUN: return "malformed name stream: string data underrun";
        case FQXV_TOK_E_PAD_UNDERRUN: return "malformed name stream: pad underrun";
        case FQXV_TOK_E_DELTA_UNDERRUN: return "malformed name stream: delta underrun";
        case FQXV_TOK_E_DELTA_PRIOR: return "malformed name stream: DELTA without numeric prior";
        case FQXV_TOK_E_UNKNOWN_OP: return "malformed name stream: unknown op";
        case FQXV_STREAM_E_CORRUPT: return "malformed lroverlap block";
        case FQXV_PERM_E_BAD: return "malformed fqxv block: bad permutation";
        case FQXV_PERM_E_LENGTH: return "malformed fqxv block: permutation length mismatch";
        default: return "unknown status";
    }
}

const char *fqxv_rans_version(void) { return "fqxv-rans-b200 0.1.0 (sm_100a)"; }

size_t fqxv_rans_encode_bound(size_t n, int order) {
    return (size_t)enc_bound_one(n, order == FQXV_RANS_ORDER0 ? FQXV_RANS_ORDER0 : FQXV_RANS_ORDER1);
}

int fqxv_rans_ctx_create(int device, fqxv_rans_ctx **out) {
    if (!out) return FQXV_RANS_E_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return FQXV_RANS_E_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return FQXV_RANS_E_INVALID_ARG;
    DeviceGuard g(device);
    auto *c = new fqxv_rans_ctx();
    c->device = device;
    c->sms = sm_count(device);
    tuning_load(c->tune, device);
    // FQXV_RANS_O1_DECODER=wide|four pins the decoder of wide order-1
    // alphabets (for measurements); anything else keeps the table's rule.
    if (const char *e = std::getenv("FQXV_RANS_O1_DECODER")) {
        if (!std::strcmp(e, "wide")) c->tune.o1_four_max_streams = 0;
        else if (!std::strcmp(e, "four")) c->tune.o1_four_max_streams = 1 << 30;
    }
    // FQXV_RANS_ENC_KEYS=0: order-1 encode without the per-position key array.
    if (const char *e = std::getenv("FQXV_RANS_ENC_KEYS")) c->tune.enc_o1_keys = std::strcmp(e, "0") != 0;
    bool ok = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) == cudaSuccess;
    // The groups of largest streams go on the highest-priority streams, so
    // their CTAs are placed before the rest of the batch fills the SMs.
    int prio_lo = 0, prio_hi = 0;
    if (cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi) != cudaSuccess) {
        cudaGetLastError();
        prio_lo = prio_hi = 0;
    }
    for (int i = 0; i < kGroups && ok; i++)
        ok = cudaStreamCreateWithPriority(&c->aux[i], cudaStreamNonBlocking,
                                          i == kGroupFourTop || i == kGroupSmallTop ? prio_hi : prio_lo) ==
                 cudaSuccess &&
             cudaEventCreateWithFlags(&c->ev_join[i], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        delete c;
        return FQXV_RANS_E_CUDA;
    }
    *out = c;
    return FQXV_RANS_OK;
}

void fqxv_rans_ctx_destroy(fqxv_rans_ctx *ctx) {
    if (!ctx) return;
    for (auto *c : ctx->sub) fqxv_rans_ctx_destroy(c);
    ctx->sub.clear();
    DeviceGuard g(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    ctx->for_each_buf([](DevBuf &b) { b.release(); });
    x_release(ctx);
    ctx->h_stage.release();
    ctx->h_io.release();
    ctx->timer.release();
    for (int i = 0; i < kGroups; i++) {
        if (ctx->aux[i]) cudaStreamDestroy(ctx->aux[i]);
        if (ctx->ev_join[i]) cudaEventDestroy(ctx->ev_join[i]);
    }
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
}

void *fqxv_rans_ctx_stream(fqxv_rans_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

uint64_t fqxv_rans_ctx_device_bytes(fqxv_rans_ctx *ctx) { return ctx ? ctx->device_bytes() : 0; }

uint64_t fqxv_rans_encode_batch_bound(const fqxv_rans_span *blocks, size_t nblocks, int order) {
    uint64_t t = 0;
    for (size_t i = 0; i < nblocks; i++) t += fqxv_rans_encode_bound(blocks[i].length, order);
    return t;
}

int fqxv_rans_encode_batch(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *blocks,
                           size_t nblocks, int order, uint8_t *d_dst, uint64_t dst_cap,
                           fqxv_rans_span *out_spans, int32_t *out_orders, int persistent) {
    if (!ctx || (nblocks && (!blocks || !out_spans || !d_dst || !d_src))) return FQXV_RANS_E_INVALID_ARG;
    std::lock_guard<std::mutex> g(ctx->mu);
    DeviceGuard dg(ctx->device);
    return encode_batch_impl(ctx, d_src, blocks, nblocks, order, d_dst, dst_cap, out_spans, out_orders,
                             persistent);
}

int fqxv_rans_decode_batch(fqxv_rans_ctx *ctx, const uint8_t *d_src, const fqxv_rans_span *blocks,
                           size_t nblocks, uint64_t max_len, uint8_t *d_dst,
                           const fqxv_rans_span *out_spans, uint64_t *out_lens, int32_t *status,
                           int persistent) {
    if (!ctx || (nblocks && (!blocks || !out_spans || !d_src))) return FQXV_RANS_E_INVALID_ARG;
    std::lock_guard<std::mutex> g(ctx->mu);
    DeviceGuard dg(ctx->device);
    return decode_batch_impl(ctx, d_src, blocks, nblocks, max_len, d_dst, out_spans, out_lens, status,
                             persistent);
}

int fqxv_rans_encode(const uint8_t *src, size_t n, int order, uint8_t *dst, size_t cap, size_t *out_len) {
    if (!out_len || !dst || (n && !src)) return FQXV_RANS_E_INVALID_ARG;
    if (order < FQXV_RANS_ORDER0 || order > FQXV_RANS_BEST_TIE1) return FQXV_RANS_E_INVALID_ARG;
    fqxv_rans_ctx *ctx;
    int st = default_ctx(&ctx);
    if (st) return st;
    std::lock_guard<std::mutex> g(ctx->mu);
    DeviceGuard dg(ctx->device);
    cudaStream_t s = ctx->stream;
    const uint64_t bound = enc_bound_one(n, order == FQXV_RANS_ORDER0 ? 0 : 1);
    CK(ctx->io_in.ensure(std::max<size_t>(n, 16), s));
    CK(ctx->io_out.ensure(bound, s));
    if (n) CK(cudaMemcpyAsync(ctx->io_in.p, src, n, cudaMemcpyHostToDevice, s));
    fqxv_rans_span blk{0, n}, out{0, 0};
    int32_t chosen = 0;
    st = encode_batch_impl(ctx, ctx->io_in.as<uint8_t>(), &blk, 1, order, ctx->io_out.as<uint8_t>(), bound, &out,
                           &chosen, 1);
    if (st) return st;
    if (out.length > cap) return FQXV_RANS_E_DST_TOO_SMALL;
    CK(cudaMemcpyAsync(dst, ctx->io_out.p, out.length, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    *out_len = out.length;
    return FQXV_RANS_OK;
}

int fqxv_rans_peek_output_len(const uint8_t *src, size_t len, uint64_t *n) {
    if (!n || (len && !src)) return FQXV_RANS_E_INVALID_ARG;
    if (len < 9) return FQXV_RANS_E_TRUNCATED;
    uint64_t v = 0;
    for (int i = 8; i >= 1; i--) v = (v << 8) | src[i];
    *n = v;
    return FQXV_RANS_OK;
}

int fqxv_rans_decode_bounded(const uint8_t *src, size_t len, size_t max_len, uint8_t *dst, size_t cap,
                             size_t *out_len) {
    if (!out_len || (len && !src)) return FQXV_RANS_E_INVALID_ARG;
    *out_len = 0;
    uint64_t n = 0;
    const bool have_n = fqxv_rans_peek_output_len(src, len, &n) == FQXV_RANS_OK;
    if (have_n && n > (uint64_t)max_len) return FQXV_RANS_E_BOUND;  // lib.rs:227, before decoding
    fqxv_rans_ctx *ctx;
    int st = default_ctx(&ctx);
    if (st) return st;
    std::lock_guard<std::mutex> g(ctx->mu);
    DeviceGuard dg(ctx->device);
    cudaStream_t s = ctx->stream;
    // Output staging only up to what the caller can take; a longer declared
    // length fails in the parse kernel with FQXV_RANS_E_ALLOC.
    const uint64_t dev_out = have_n ? std::min<uint64_t>(n, cap) : 0;
    if (dev_out && !dst) return FQXV_RANS_E_INVALID_ARG;
    CK(ctx->io_in.ensure(std::max<size_t>(len, 16), s));
    CK(ctx->io_out.ensure(std::max<uint64_t>(dev_out, 16), s));
    if (len) CK(cudaMemcpyAsync(ctx->io_in.p, src, len, cudaMemcpyHostToDevice, s));
    fqxv_rans_span blk{0, len}, out{0, cap};
    uint64_t olen = 0;
    int32_t bst = 0;
    st = decode_batch_impl(ctx, ctx->io_in.as<uint8_t>(), &blk, 1, UINT64_MAX, ctx->io_out.as<uint8_t>(), &out,
                           &olen, &bst, 1);
    if (st) return st;
    if (olen) {
        CK(cudaMemcpyAsync(dst, ctx->io_out.p, olen, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
    }
    *out_len = olen;
    return FQXV_RANS_OK;
}

int fqxv_rans_decode(const uint8_t *src, size_t len, uint8_t *dst, size_t cap, size_t *out_len) {
    return fqxv_rans_decode_bounded(src, len, SIZE_MAX, dst, cap, out_len);
}

int fqxv_rans_decode_with(const uint8_t *src, size_t len, int backend, uint8_t *dst, size_t cap,
                          size_t *out_len) {
    (void)backend;  // lib.rs:241-255: every backend yields the same output
    return fqxv_rans_decode(src, len, dst, cap, out_len);
}

int fqxv_rans_ctx_set_profiling(fqxv_rans_ctx *ctx, int on) {
    if (!ctx) return FQXV_RANS_E_INVALID_ARG;
    std::lock_guard<std::mutex> g(ctx->mu);
    ctx->timer.on = on != 0;
    return FQXV_RANS_OK;
}

int fqxv_rans_ctx_set_param(fqxv_rans_ctx *ctx, const char *name, int64_t value) {
    if (!ctx || !name) return FQXV_RANS_E_INVALID_ARG;
    std::lock_guard<std::mutex> g(ctx->mu);
    const int st = tuning_set(ctx->tune, name, value);
    if (st == FQXV_RANS_OK)
        for (auto *c : ctx->sub) tuning_set(c->tune, name, value);
    return st;
}

int fqxv_rans_ctx_get_param(fqxv_rans_ctx *ctx, const char *name, int64_t *value) {
    if (!ctx || !name || !value) return FQXV_RANS_E_INVALID_ARG;
    std::lock_guard<std::mutex> g(ctx->mu);
    return tuning_get(ctx->tune, name, *value);
}

const char *fqxv_rans_ctx_tuning_source(fqxv_rans_ctx *ctx) {
    return ctx && !ctx->tune.source.empty() ? ctx->tune.source.c_str() : "";
}

int fqxv_rans_ctx_test_set_wait_polls(fqxv_rans_ctx *ctx, uint32_t polls) {
    if (!ctx) return FQXV_RANS_E_INVALID_ARG;
    std::lock_guard<std::mutex> g(ctx->mu);
    ctx->first_polls = polls;
    for (auto *c : ctx->sub) c->first_polls = ctx->first_polls;
    return FQXV_RANS_OK;
}

int fqxv_rans_ctx_stage_stats(fqxv_rans_ctx *ctx, fqxv_rans_stage_stat *out, int cap, int *n, int reset) {
    if (!ctx || !n || (cap > 0 && !out)) return FQXV_RANS_E_INVALID_ARG;
    std::lock_guard<std::mutex> g(ctx->mu);
    int k = 0;
    for (int i = 0; i < kStages && k < cap; i++, k++) {
        std::memset(out[k].name, 0, sizeof out[k].name);
        std::strncpy(out[k].name, kStageNames[i], sizeof out[k].name - 1);
        out[k].launches = ctx->timer.launches[i];
        out[k].ms = ctx->timer.ms[i];
        out[k].bytes = ctx->timer.bytes[i];
        out[k].wall_ms = ctx->timer.wall_ms[i];
        out[k].ctas_per_sm = ctx->timer.ctas_per_sm[i];
        out[k].smem_bytes = ctx->timer.smem_bytes[i];
    }
    *n = k;
    if (reset) {
        for (int i = 0; i < kStages; i++) {
            ctx->timer.launches[i] = 0;
            ctx->timer.ms[i] = 0.0;
            ctx->timer.wall_ms[i] = 0.0;
            ctx->timer.bytes[i] = 0;
            ctx->timer.ctas_per_sm[i] = 0;
            ctx->timer.smem_bytes[i] = 0;
        }
    }
    return FQXV_RANS_OK;
}

}  // extern "C"

namespace {

// Encode on one context: input copied in, coded, and -- once `place` gives
// where this batch's streams go in h_dst (it may wait for an earlier chunk)
// -- copied out. Offsets of out_spans are local to the batch on entry to
// `place` and final on return.
// `gate(s, before)` runs on the batch's stream right before (before = true)
// and after its input copy is issued, so that chunks can order their copies.
struct NoGate {
    void operator()(cudaStream_t, bool) const {}
};
template <class Place, class Gate = NoGate>
int encode_host_one(fqxv_rans_ctx *ctx, const uint8_t *h_src, const fqxv_rans_span *blocks, size_t nblocks,
                    int order, fqxv_rans_span *out_spans, int32_t *out_orders, Place &&place, Gate &&gate = Gate()) {
    DeviceGuard dg(ctx->device);
    cudaStream_t s = ctx->stream;
    uint64_t end = 0;
    for (size_t i = 0; i < nblocks; i++) end = std::max<uint64_t>(end, blocks[i].offset + blocks[i].length);
    const uint64_t bound = fqxv_rans_encode_batch_bound(blocks, nblocks, order);
    CK(ctx->io_in.ensure(std::max<uint64_t>(end, 16), s));
    CK(ctx->io_out.ensure(std::max<uint64_t>(bound, 16), s));
    gate(s, true);
    const cudaError_t ce = cudaMemcpyAsync(ctx->io_in.p, h_src, end, cudaMemcpyHostToDevice, s);
    gate(s, false);
    CK(ce);
    int st = encode_batch_impl(ctx, ctx->io_in.as<uint8_t>(), blocks, nblocks, order, ctx->io_out.as<uint8_t>(),
                               bound, out_spans, out_orders, 1);
    const uint64_t total = st ? 0 : out_spans[nblocks - 1].offset + out_spans[nblocks - 1].length;
    uint8_t *dst = nullptr;
    const int pst = place(st, total, dst);  // publishes this batch's end for the next chunk
    if (st) return st;
    if (pst) return pst;
    CK(cudaMemcpyAsync(dst, ctx->io_out.p, total, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return FQXV_RANS_OK;
}

// Host-buffer batches of at least kPipeMinBytes are cut into up to
// `host_enc_chunks` (encode) or `host_dec_chunks` (decode) chunks of
// consecutive blocks, each coded by its own sub-context on its own host
// thread: one chunk's copies overlap the other chunks' kernels.
constexpr uint64_t kPipeMinBytes = 32ull << 20;

// [first, last) block ranges of roughly equal bytes
std::vector<std::pair<size_t, size_t>> pipe_chunks(const fqxv_rans_span *blocks, size_t n, int64_t nchunks) {
    std::vector<std::pair<size_t, size_t>> out;
    uint64_t total = 0;
    for (size_t i = 0; i < n; i++) total += blocks[i].length;
    if (total < kPipeMinBytes || n < 2) {
        out.emplace_back(0, n);
        return out;
    }
    const int k = (int)std::min<size_t>((size_t)std::max<int64_t>(nchunks, 1), n);
    size_t b = 0;
    uint64_t acc = 0;
    for (int c = 0; c < k && b < n; c++) {
        const uint64_t target = total * (uint64_t)(c + 1) / (uint64_t)k;
        size_t e = b + 1;
        acc += blocks[b].length;
        while (e < n && (c == k - 1 || acc + blocks[e].length <= target)) acc += blocks[e++].length;
        out.emplace_back(b, e);
        b = e;
    }
    if (b < n) out.back().second = n;
    return out;
}

// The sub-contexts of a context (created on first use, same device).
int ensure_subs(fqxv_rans_ctx *ctx, size_t k) {
    while (ctx->sub.size() < k) {
        fqxv_rans_ctx *c = nullptr;
        const int st = fqxv_rans_ctx_create(ctx->device, &c);
        if (st != FQXV_RANS_OK) return st;
        c->first_polls = ctx->first_polls;
        c->tune = ctx->tune;
        ctx->sub.push_back(c);
    }
    return FQXV_RANS_OK;
}

// Rebased copy of spans [b, e): offsets relative to the first byte any of
// them touches; returns that byte's offset.
uint64_t rebase(const fqxv_rans_span *spans, size_t b, size_t e, std::vector<fqxv_rans_span> &out) {
    uint64_t lo = UINT64_MAX;
    for (size_t i = b; i < e; i++) lo = std::min<uint64_t>(lo, spans[i].offset);
    if (lo == UINT64_MAX) lo = 0;
    out.resize(e - b);
    for (size_t i = b; i < e; i++) out[i - b] = {spans[i].offset - lo, spans[i].length};
    return lo;
}

}  // namespace

extern "C" {

int fqxv_rans_encode_batch_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, const fqxv_rans_span *blocks,
                                size_t nblocks, int order, uint8_t *h_dst, uint64_t dst_cap,
                                fqxv_rans_span *out_spans, int32_t *out_orders) {
    if (!ctx || (nblocks && (!blocks || !out_spans || !h_dst || !h_src))) return FQXV_RANS_E_INVALID_ARG;
    if (order < FQXV_RANS_ORDER0 || order > FQXV_RANS_BEST_TIE1) return FQXV_RANS_E_INVALID_ARG;
    if (nblocks == 0) return FQXV_RANS_OK;
    NvtxRange range("fqxv.encode_batch_host");
    std::lock_guard<std::mutex> g(ctx->mu);
    const auto chunks = pipe_chunks(blocks, nblocks, ctx->tune.host_enc_chunks);
    if (chunks.size() == 1) {
        return encode_host_one(ctx, h_src, blocks, nblocks, order, out_spans, out_orders,
                               [&](int st, uint64_t total, uint8_t *&dst) -> int {
                                   if (st) return st;
                                   if (total > dst_cap) return FQXV_RANS_E_DST_TOO_SMALL;
                                   dst = h_dst;
                                   return FQXV_RANS_OK;
                               });
    }
    const size_t k = chunks.size();
    int cst = ensure_subs(ctx, k);
    if (cst != FQXV_RANS_OK) return cst;
    // chunk c's streams follow chunk c-1's: each chunk publishes where its
    // output ends as soon as its encode is done, before its own copy out
    std::mutex pm;
    std::condition_variable pcv;
    std::vector<uint64_t> ends(k + 1, 0);
    std::vector<int> ready(k + 1, 0), sts(k, FQXV_RANS_OK);
    ready[0] = 1;
    bool failed = false;
    // The chunks' input copies go one after another in chunk order (each
    // chunk's copy waits on the previous one's), so the first chunk's
    // encode starts after a quarter of the input has crossed the host link
    // instead of after all of it.
    std::vector<cudaEvent_t> copied(k, nullptr);
    for (size_t c = 0; c < k; c++)
        if (cudaEventCreateWithFlags(&copied[c], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            copied[c] = nullptr;
        }
    std::vector<int> issued(k + 1, 0);
    issued[0] = 1;
    std::vector<std::thread> th;
    for (size_t c = 0; c < k; c++) {
        th.emplace_back([&, c] {
            const size_t b = chunks[c].first, e = chunks[c].second;
            std::vector<fqxv_rans_span> local;
            const uint64_t lo = rebase(blocks, b, e, local);
            sts[c] = encode_host_one(ctx->sub[c], h_src + lo, local.data(), e - b, order, out_spans + b,
                                     out_orders + b, [&, c](int st, uint64_t total, uint8_t *&dst) -> int {
                                         std::unique_lock<std::mutex> lk(pm);
                                         pcv.wait(lk, [&] { return ready[c] != 0; });
                                         int r = FQXV_RANS_OK;
                                         if (st || failed) {
                                             failed = true;
                                             r = st ? st : FQXV_RANS_E_INVALID_ARG;
                                         } else if (ends[c] + total > dst_cap) {
                                             failed = true;
                                             r = FQXV_RANS_E_DST_TOO_SMALL;
                                         } else {
                                             dst = h_dst + ends[c];
                                             for (size_t i = b; i < e; i++) out_spans[i].offset += ends[c];
                                             ends[c + 1] = ends[c] + total;
                                         }
                                         ready[c + 1] = 1;
                                         pcv.notify_all();
                                         return r;
                                     },
                                     [&, c](cudaStream_t s, bool before) {
                                         std::unique_lock<std::mutex> lk(pm);
                                         if (before) {
                                             pcv.wait(lk, [&] { return issued[c] != 0; });
                                             if (c > 0 && copied[c - 1]) cudaStreamWaitEvent(s, copied[c - 1], 0);
                                         } else {
                                             if (copied[c]) cudaEventRecord(copied[c], s);
                                             issued[c + 1] = 1;
                                             pcv.notify_all();
                                         }
                                     });
            // a chunk that stopped before placing its output (a failed copy
            // or allocation) still releases the chunks after it
            std::lock_guard<std::mutex> lk(pm);
            if (!ready[c + 1]) {
                failed = true;
                ready[c + 1] = 1;
            }
            issued[c + 1] = 1;
            pcv.notify_all();
        });
    }
    for (auto &t : th) t.join();
    for (cudaEvent_t e : copied)
        if (e) cudaEventDestroy(e);
    // the first failing chunk in block order decides (a later chunk that only
    // stopped because an earlier one failed reports that one's status)
    for (size_t c = 0; c < k; c++)
        if (sts[c] != FQXV_RANS_OK) return sts[c];
    return FQXV_RANS_OK;
}

}  // extern "C"

namespace {

// Decode on one context (the caller holds its lock).
int decode_host_one(fqxv_rans_ctx *ctx, const uint8_t *h_src, const fqxv_rans_span *blocks, size_t nblocks,
                    uint64_t max_len, uint8_t *h_dst, const fqxv_rans_span *out_spans, uint64_t *out_lens,
                    int32_t *status) {
    DeviceGuard dg(ctx->device);
    cudaStream_t s = ctx->stream;
    uint64_t end = 0, oend = 0;
    for (size_t i = 0; i < nblocks; i++) {
        end = std::max<uint64_t>(end, blocks[i].offset + blocks[i].length);
        oend = std::max<uint64_t>(oend, out_spans[i].offset + out_spans[i].length);
    }
    // The compressed input of a batch of fewer than kZeroCopyMinStreams
    // streams is staged by one copy, issued first (the decoders' word reads
    // are latency-sensitive). A pinned (mapped) destination of a large batch
    // is mirrored: the kernels decode into device memory and the CTA that
    // finished a stream copies it to the destination in 16-byte stores
    // while other streams still decode, so the output transfer overlaps the
    // decode instead of following it. Other destinations are staged and
    // copied once the batch is done.
    const uint8_t *d_in = nullptr;
    auto stage_input = [&]() -> cudaError_t {
        cudaError_t e = ctx->io_in.ensure(std::max<uint64_t>(end, 16), s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->io_in.p, h_src, end, cudaMemcpyHostToDevice, s);
        d_in = ctx->io_in.as<uint8_t>();
        return e;
    };
    const int64_t in_place = ctx->tune.host_in_place;
    if (in_place == 0 || (in_place < 0 && nblocks < kZeroCopyMinStreams)) CK(stage_input());
    uint8_t *mirror = oend >= kZeroCopyMinBytes && ctx->tune.host_out_mirror
                          ? static_cast<uint8_t *>(mapped_device_ptr(h_dst))
                          : nullptr;
    // A slow batch of hundreds of streams also reads its pinned input in
    // place: each stream's words are fetched 16 bytes a lane, segments ahead
    // of use, at a small share of the link, and the decode starts without
    // waiting for a copy. Measured on B200: 4103 mixed streams (4 KiB to
    // 4 MiB) e2e 17.2 -> 21.2 GB/s, but chunks of 16 x 1 MiB order-1 streams
    // 4.63 -> 4.36, so smaller batches (and single serving requests) keep
    // the staged copy, issued before this point. "Slow": the decode time,
    // estimated from the stream headers (the largest stream's serial rounds,
    // about 320 ns per 32 bytes for order-1 and 80 ns for order-0 on B200,
    // or the whole batch at the batched rates, about 15 and 300 GB/s), keeps
    // the output rate under 40 GB/s.
    if (!d_in && in_place > 0) d_in = static_cast<const uint8_t *>(mapped_device_ptr(h_src));
    if (!d_in && mirror) {
        double t_lat = 0.0, b0 = 0.0, b1 = 0.0;
        for (size_t i = 0; i < nblocks; i++) {
            if (blocks[i].length < kHdr) continue;
            const uint8_t *h = h_src + blocks[i].offset;
            uint64_t n = 0;
            for (int k = 0; k < 8; k++) n |= (uint64_t)h[1 + k] << (8 * k);
            if (n > out_spans[i].length) continue;
            const bool o1 = h[0] == 1;
            t_lat = std::max(t_lat, (double)(n / 32) * (o1 ? 320e-9 : 80e-9));
            (o1 ? b1 : b0) += (double)n;
        }
        const double t_est = std::max(t_lat, b1 / 15e9 + b0 / 300e9);
        if (t_est > 0.0 && (double)oend / t_est < 40e9)
            d_in = static_cast<const uint8_t *>(mapped_device_ptr(h_src));
    }
    if (!d_in) CK(stage_input());
    // the staging buffer sits at the destination's address modulo 16, so a
    // stream's staged and final bytes are congruent (16-byte stores)
    const uint64_t skew = mirror ? (uint64_t)((uintptr_t)h_dst & 15u) : 0u;
    CK(ctx->io_out.ensure(std::max<uint64_t>(oend + skew, 16), s));
    uint8_t *d_out = ctx->io_out.as<uint8_t>() + skew;
    std::vector<uint64_t> lens(nblocks);
    std::vector<int32_t> sts(nblocks);
    const int first = decode_batch_impl(ctx, d_in, blocks, nblocks, max_len, d_out, out_spans, lens.data(),
                                        sts.data(), 1, mirror);
    if (first != FQXV_RANS_OK && (first < FQXV_RANS_E_TRUNCATED || first > FQXV_RANS_E_TRUNCATED_RENORM))
        return first;
    if (mirror) {
        for (size_t i = 0; i < nblocks; i++) {
            if (out_lens) out_lens[i] = lens[i];
            if (status) status[i] = sts[i];
        }
        return first;
    }
    // One copy of the whole output range when the spans are dense, else one
    // copy per decoded block.
    uint64_t produced = 0;
    for (size_t i = 0; i < nblocks; i++) produced += lens[i];
    if (produced == oend && first == FQXV_RANS_OK) {
        CK(cudaMemcpyAsync(h_dst, d_out, oend, cudaMemcpyDeviceToHost, s));
    } else {
        for (size_t i = 0; i < nblocks; i++)
            if (lens[i])
                CK(cudaMemcpyAsync(h_dst + out_spans[i].offset, d_out + out_spans[i].offset, lens[i],
                                   cudaMemcpyDeviceToHost, s));
    }
    CK(cudaStreamSynchronize(s));
    for (size_t i = 0; i < nblocks; i++) {
        if (out_lens) out_lens[i] = lens[i];
        if (status) status[i] = sts[i];
    }
    return first;
}

}  // namespace

extern "C" {

int fqxv_rans_decode_batch_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, const fqxv_rans_span *blocks,
                                size_t nblocks, uint64_t max_len, uint8_t *h_dst,
                                const fqxv_rans_span *out_spans, uint64_t *out_lens, int32_t *status) {
    if (!ctx || (nblocks && (!blocks || !out_spans || !h_src || !h_dst))) return FQXV_RANS_E_INVALID_ARG;
    if (nblocks == 0) return FQXV_RANS_OK;
    NvtxRange range("fqxv.decode_batch_host");
    std::lock_guard<std::mutex> g(ctx->mu);
    const auto chunks = pipe_chunks(blocks, nblocks, ctx->tune.host_dec_chunks);
    if (chunks.size() == 1)
        return decode_host_one(ctx, h_src, blocks, nblocks, max_len, h_dst, out_spans, out_lens, status);
    const size_t k = chunks.size();
    const int cst = ensure_subs(ctx, k);
    if (cst != FQXV_RANS_OK) return cst;
    std::vector<int> firsts(k, FQXV_RANS_OK);
    std::vector<std::thread> th;
    for (size_t c = 0; c < k; c++) {
        th.emplace_back([&, c] {
            const size_t b = chunks[c].first, e = chunks[c].second;
            std::vector<fqxv_rans_span> lin, lout;
            const uint64_t lo = rebase(blocks, b, e, lin);
            const uint64_t olo = rebase(out_spans, b, e, lout);
            firsts[c] = decode_host_one(ctx->sub[c], h_src + lo, lin.data(), e - b, max_len, h_dst + olo,
                                        lout.data(), out_lens ? out_lens + b : nullptr,
                                        status ? status + b : nullptr);
        });
    }
    for (auto &t : th) t.join();
    // a device failure anywhere wins; otherwise the first malformed stream
    for (size_t c = 0; c < k; c++)
        if (firsts[c] != FQXV_RANS_OK && (firsts[c] < FQXV_RANS_E_TRUNCATED || firsts[c] > FQXV_RANS_E_TRUNCATED_RENORM))
            return firsts[c];
    for (size_t c = 0; c < k; c++)
        if (firsts[c] != FQXV_RANS_OK) return firsts[c];
    return FQXV_RANS_OK;
}

}  // extern "C"
