// Serving runtime: requests arrive one at a time (compress or decompress of
// one stream), are admitted while their device-memory estimate fits under a
// cap, and are coded in continuous batches: every worker owns a context (its
// own CUDA stream, device arenas and pinned staging); whenever a worker is
// free it takes all admitted requests that share the oldest request's kind,
// order mode and size class (sizes within a factor of four) and runs them as
// one batched pass, so requests that arrive while others are on the GPU join
// the next pass of any free worker, passes of different workers overlap on
// the device, and a small request never waits for a large one in its own
// pass. One stream is coded serially (its 32 states advance round by round),
// so a request's latency is at least its own stream's; the runtime only
// keeps queueing from adding to it. No reference counterpart (the reference
// is a library called per stream); results are byte-identical to the single
// calls.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "rans_internal.cuh"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id = 0;
    int kind = 0;          // 0 encode, 1 decode
    int size_class = 0;    // floor(log4(input bytes))
    int order = 0;         // encode order mode
    uint64_t max_len = 0;  // decode bound
    std::vector<uint8_t> in;
    std::vector<uint8_t> out;
    uint64_t n_out = 0;    // decode: declared output length (capacity)
    uint64_t mem = 0;      // admission estimate (device bytes)
    int status = FQXV_RANS_OK;
    bool done = false;
    Clock::time_point t_submit, t_done;
};

struct HostPinned {
    void *p = nullptr;
    size_t cap = 0;
    bool ensure(size_t want) {
        if (want <= cap) return true;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        size_t nc = std::max(want, 2 * cap) + (1 << 20);
        if (cudaHostAlloc(&p, nc, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        cap = nc;
        return true;
    }
    ~HostPinned() {
        if (p) cudaFreeHost(p);
    }
};

int size_class(size_t n) {
    int b = 0;
    while (n > 1) {
        n >>= 1;
        b++;
    }
    return b / 2;
}

uint64_t request_mem(const Request &r) {
    // Inputs, outputs and the per-block scratch of the batched passes.
    if (r.kind == 0) {
        const uint64_t n = r.in.size();
        return n + fqxv_rans_encode_bound(n, r.order) + 6 * n + fqxv::enc_table_bytes(n) + (1 << 16);
    }
    return r.in.size() + r.n_out + fqxv::dec_table_bytes(r.in.size()) + (1 << 16);
}

}  // namespace

struct fqxv_rans_server {
    int device = 0;
    uint64_t cap = 0;
    uint64_t in_use = 0, peak = 0;
    uint64_t next_id = 1;
    uint64_t completed = 0, batches = 0;
    size_t max_batch_bytes = 1ull << 30;
    bool stop = false;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> pending;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> all;
    std::vector<fqxv_rans_ctx *> ctxs;
    std::vector<std::thread> workers;
    int warmed = 0;

    void worker(int w);
};

namespace {

// Bring a worker to serving state before the first request: pinned staging
// of a useful size, and one small pass of each kernel path (order-0 and
// order-1 encode and decode) so module loading, kernel attributes and the
// context's device arenas are in place.
void warm_worker(fqxv_rans_ctx *ctx, HostPinned &h_in, HostPinned &h_out) {
    const size_t n = 1 << 16;
    // 64 MiB each way covers a request of the largest usual size without
    // pinning more memory on the request path (pinning costs about half a
    // millisecond per MiB); larger batches grow the buffers geometrically.
    if (!h_in.ensure(64u << 20) || !h_out.ensure(64u << 20)) return;
    uint8_t *src = static_cast<uint8_t *>(h_in.p);
    uint32_t z = 12345;
    for (size_t i = 0; i < n; i++) {
        z = z * 1103515245u + 12345u;
        src[i] = (uint8_t)('A' + ((z >> 16) % 5));
    }
    uint8_t *enc = static_cast<uint8_t *>(h_out.p);
    uint8_t *dec = src + n;
    for (int order = FQXV_RANS_ORDER0; order <= FQXV_RANS_ORDER1; order++) {
        fqxv_rans_span sp{0, n}, out{0, 0}, dsp{0, n};
        int32_t ord = 0, st = 0;
        uint64_t len = 0;
        const uint64_t bound = fqxv_rans_encode_batch_bound(&sp, 1, order);
        if (fqxv_rans_encode_batch_host(ctx, src, &sp, 1, order, enc, bound, &out, &ord) != FQXV_RANS_OK) return;
        fqxv_rans_decode_batch_host(ctx, enc, &out, 1, n, dec, &dsp, &len, &st);
    }
}

}  // namespace

void fqxv_rans_server::worker(int w) {
    cudaSetDevice(device);
    fqxv_rans_ctx *ctx = ctxs[w];
    HostPinned h_in, h_out;
    warm_worker(ctx, h_in, h_out);
    {
        std::lock_guard<std::mutex> lk(mu);
        warmed++;
    }
    cv_done.notify_all();
    std::vector<Request *> batch;
    std::vector<fqxv_rans_span> spans, outs;
    std::vector<int32_t> orders, sts;
    std::vector<uint64_t> lens;
    for (;;) {
        batch.clear();
        uint64_t bmem = 0;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait(lk, [&] {
                if (stop) return true;
                if (pending.empty()) return false;
                const Request *h = pending.front();
                return in_use == 0 || in_use + h->mem <= cap;
            });
            if (stop && pending.empty()) return;
            if (pending.empty()) continue;
            const int kind = pending.front()->kind, order = pending.front()->order;
            const int cls = pending.front()->size_class;
            size_t bytes = 0;
            // Continuous batching: everything admissible of the head's shape.
            for (auto it = pending.begin(); it != pending.end();) {
                Request *r = *it;
                const bool same = r->kind == kind && r->size_class == cls && (kind == 1 || r->order == order);
                const bool fits = (in_use + bmem == 0) || in_use + bmem + r->mem <= cap;
                if (same && fits && (batch.empty() || bytes + r->in.size() <= max_batch_bytes)) {
                    batch.push_back(r);
                    bmem += r->mem;
                    bytes += r->in.size();
                    it = pending.erase(it);
                } else if (!fits) {
                    break;  // admission in arrival order
                } else {
                    ++it;
                }
            }
            in_use += bmem;
            if (in_use > peak) peak = in_use;
        }
        const size_t nb = batch.size();
        spans.resize(nb);
        outs.resize(nb);
        orders.resize(nb);
        sts.resize(nb);
        lens.resize(nb);
        uint64_t tin = 0, tout = 0;
        for (size_t i = 0; i < nb; i++) {
            spans[i] = {tin, batch[i]->in.size()};
            tin += batch[i]->in.size();
        }
        int st = FQXV_RANS_OK;
        if (!h_in.ensure(tin + 16)) st = FQXV_RANS_E_OUT_OF_MEMORY;
        if (st == FQXV_RANS_OK) {
            for (size_t i = 0; i < nb; i++)
                if (!batch[i]->in.empty())
                    std::memcpy((uint8_t *)h_in.p + spans[i].offset, batch[i]->in.data(), batch[i]->in.size());
            if (batch[0]->kind == 0) {
                tout = fqxv_rans_encode_batch_bound(spans.data(), nb, batch[0]->order);
                if (!h_out.ensure(tout + 16)) st = FQXV_RANS_E_OUT_OF_MEMORY;
                if (st == FQXV_RANS_OK)
                    st = fqxv_rans_encode_batch_host(ctx, (const uint8_t *)h_in.p, spans.data(), nb,
                                                     batch[0]->order, (uint8_t *)h_out.p, tout, outs.data(),
                                                     orders.data());
                for (size_t i = 0; i < nb; i++) sts[i] = st;
                if (st == FQXV_RANS_OK)
                    for (size_t i = 0; i < nb; i++)
                        batch[i]->out.assign((uint8_t *)h_out.p + outs[i].offset,
                                             (uint8_t *)h_out.p + outs[i].offset + outs[i].length);
            } else {
                for (size_t i = 0; i < nb; i++) {
                    outs[i] = {tout, batch[i]->n_out};
                    tout += batch[i]->n_out;
                }
                if (!h_out.ensure(tout + 16)) st = FQXV_RANS_E_OUT_OF_MEMORY;
                uint64_t max_len = 0;
                for (size_t i = 0; i < nb; i++) max_len = std::max(max_len, batch[i]->max_len);
                if (st == FQXV_RANS_OK) {
                    // Every member's declared length was checked against its
                    // own bound at submission, so the pass may use the largest.
                    const int first = fqxv_rans_decode_batch_host(ctx, (const uint8_t *)h_in.p, spans.data(), nb,
                                                                  max_len, (uint8_t *)h_out.p,
                                                                  outs.data(), lens.data(), sts.data());
                    if (first > FQXV_RANS_E_TRUNCATED_RENORM) {
                        for (size_t i = 0; i < nb; i++) sts[i] = first;
                    } else {
                        for (size_t i = 0; i < nb; i++)
                            if (sts[i] == FQXV_RANS_OK)
                                batch[i]->out.assign((uint8_t *)h_out.p + outs[i].offset,
                                                     (uint8_t *)h_out.p + outs[i].offset + lens[i]);
                    }
                } else {
                    for (size_t i = 0; i < nb; i++) sts[i] = st;
                }
            }
        }
        {
            std::lock_guard<std::mutex> lk(mu);
            const auto now = Clock::now();
            for (size_t i = 0; i < nb; i++) {
                batch[i]->status = sts[i];
                batch[i]->done = true;
                batch[i]->t_done = now;
                std::vector<uint8_t>().swap(batch[i]->in);
            }
            in_use -= bmem;
            completed += nb;
            batches++;
        }
        cv_done.notify_all();
        cv_work.notify_all();
    }
}

extern "C" {

int fqxv_rans_server_create(int device, int n_workers, uint64_t hbm_cap, fqxv_rans_server **out) {
    if (!out || n_workers < 1 || n_workers > 64) return FQXV_RANS_E_INVALID_ARG;
    *out = nullptr;
    auto *s = new fqxv_rans_server();
    s->device = device;
    s->cap = hbm_cap ? hbm_cap : (40ull << 30);
    for (int i = 0; i < n_workers; i++) {
        fqxv_rans_ctx *c = nullptr;
        const int st = fqxv_rans_ctx_create(device, &c);
        if (st != FQXV_RANS_OK) {
            for (auto *x : s->ctxs) fqxv_rans_ctx_destroy(x);
            delete s;
            return st;
        }
        // Workers decode their batches side by side on one GPU: a batch's
        // top groups must not claim SMs of their own there, or each worker's
        // CTAs wait for SMs the others hold (config4's capacity, measured on
        // B200: 0.16-0.18 GB/s with them, 0.23-0.29 without).
        fqxv_rans_ctx_set_param(c, "o1_top_exclusive", 0);
        s->ctxs.push_back(c);
    }
    for (int i = 0; i < n_workers; i++) s->workers.emplace_back([s, i] { s->worker(i); });
    {
        std::unique_lock<std::mutex> lk(s->mu);
        s->cv_done.wait(lk, [&] { return s->warmed == n_workers; });
    }
    *out = s;
    return FQXV_RANS_OK;
}

void fqxv_rans_server_destroy(fqxv_rans_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto &t : s->workers) t.join();
    for (auto *c : s->ctxs) fqxv_rans_ctx_destroy(c);
    delete s;
}

int fqxv_rans_server_submit(fqxv_rans_server *s, int kind, const uint8_t *src, size_t len, int order,
                            uint64_t max_len, uint64_t *id) {
    if (!s || !id || (len && !src) || (kind != 0 && kind != 1)) return FQXV_RANS_E_INVALID_ARG;
    if (kind == 0 && (order < FQXV_RANS_ORDER0 || order > FQXV_RANS_BEST_TIE1)) return FQXV_RANS_E_INVALID_ARG;
    auto r = std::make_unique<Request>();
    r->kind = kind;
    r->order = kind == 0 ? order : 0;
    r->max_len = kind == 1 ? max_len : 0;
    r->in.assign(src, src + len);
    r->size_class = size_class(len);
    bool bound_exceeded = false;
    if (kind == 1) {
        uint64_t n = 0;
        // A stream too short for a header decodes to an error; reserve nothing.
        if (fqxv_rans_peek_output_len(src, len, &n) == FQXV_RANS_OK) {
            if (n <= max_len) r->n_out = n;
            else bound_exceeded = true;  // lib.rs:227: rejected before decoding
        }
    }
    r->mem = request_mem(*r);
    if (r->mem > s->cap) return FQXV_RANS_E_TOO_LARGE;
    r->t_submit = Clock::now();
    if (bound_exceeded) {
        std::lock_guard<std::mutex> lk(s->mu);
        r->id = s->next_id++;
        *id = r->id;
        r->status = FQXV_RANS_E_BOUND;
        r->done = true;
        r->t_done = r->t_submit;
        std::vector<uint8_t>().swap(r->in);
        s->completed++;
        s->all.emplace(r->id, std::move(r));
        s->cv_done.notify_all();
        return FQXV_RANS_OK;
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->id = s->next_id++;
        *id = r->id;
        s->pending.push_back(r.get());
        s->all.emplace(r->id, std::move(r));
    }
    s->cv_work.notify_one();
    return FQXV_RANS_OK;
}

int fqxv_rans_server_wait(fqxv_rans_server *s, uint64_t id, int timeout_ms, size_t *out_len, int32_t *status,
                          double *latency_us) {
    if (!s) return FQXV_RANS_E_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return FQXV_RANS_E_INVALID_ARG;
    Request *r = it->second.get();
    auto ready = [&] { return r->done; };
    if (timeout_ms < 0) s->cv_done.wait(lk, ready);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return FQXV_RANS_E_TIMEOUT;
    if (out_len) *out_len = r->out.size();
    if (status) *status = r->status;
    if (latency_us)
        *latency_us = std::chrono::duration<double, std::micro>(r->t_done - r->t_submit).count();
    return FQXV_RANS_OK;
}

int fqxv_rans_server_take(fqxv_rans_server *s, uint64_t id, uint8_t *dst, size_t cap) {
    if (!s) return FQXV_RANS_E_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end() || !it->second->done) return FQXV_RANS_E_INVALID_ARG;
    Request *r = it->second.get();
    if (r->out.size() > cap) return FQXV_RANS_E_DST_TOO_SMALL;
    if (!r->out.empty()) std::memcpy(dst, r->out.data(), r->out.size());
    s->all.erase(it);
    return FQXV_RANS_OK;
}

int fqxv_rans_server_stats(fqxv_rans_server *s, uint64_t *completed, uint64_t *batches, uint64_t *peak_bytes,
                           uint64_t *pending) {
    if (!s) return FQXV_RANS_E_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    if (completed) *completed = s->completed;
    if (batches) *batches = s->batches;
    if (peak_bytes) *peak_bytes = s->peak;
    if (pending) *pending = s->pending.size();
    return FQXV_RANS_OK;
}

}  // extern "C"
