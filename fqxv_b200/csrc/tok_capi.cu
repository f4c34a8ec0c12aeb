// Read-name tokenizer of crates/fqxv-tokenizer/src/lib.rs over the batched
// GPU coder (include/fqxv_tok_gpu.h). Tokenising names into role streams and
// rebuilding names from them is serial per block and runs on host threads,
// one block per thread; every role stream of every block is rANS-coded or
// decoded in one pass of the batch kernels (fqxv_rans_encode_batch_host /
// fqxv_rans_decode_batch_host).
#include <algorithm>
#include <atomic>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fqxv_tok_gpu.h"

namespace {

// lib.rs:54-75
constexpr uint8_t kVersion = 1;
constexpr uint8_t kMatch = 0, kStr = 1, kNum = 2, kDelta = 3;
constexpr size_t kMaxNumDigits = 18;
constexpr int kCols = 64;  // MAX_COL + 1
constexpr uint64_t kMaxExpansion = 1ull << 16;
constexpr uint64_t kMinStreamBound = 1ull << 20;
// The eight flat / op-run streams of a payload, in payload order.
constexpr int kFlat = 8;

void put_varint(std::vector<uint8_t> &out, uint64_t v) {  // fqxv-bytes lib.rs:14-24
    for (;;) {
        const uint8_t b = (uint8_t)(v & 0x7F);
        v >>= 7;
        if (!v) {
            out.push_back(b);
            return;
        }
        out.push_back(b | 0x80);
    }
}

uint64_t zigzag(int64_t d) { return ((uint64_t)d << 1) ^ (uint64_t)(d >> 63); }
int64_t unzigzag(uint64_t z) { return (int64_t)((z >> 1) ^ (0 - (z & 1))); }

template <class F>
void parallel_for(size_t n, F &&f) {
    size_t nt = std::min<size_t>(n, std::max(1u, std::min(32u, std::thread::hardware_concurrency())));
    if (nt <= 1) {
        for (size_t i = 0; i < n; i++) f(i);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> th;
    for (size_t t = 0; t < nt; t++)
        th.emplace_back([&] {
            for (size_t i; (i = next.fetch_add(1)) < n;) f(i);
        });
    for (auto &t : th) t.join();
}

// ---- encode (lib.rs:482-540) ----------------------------------------------------

struct Tok {
    const uint8_t *p;
    uint32_t len;
    bool is_num;
    int64_t value;
};

// lib.rs:654-680: maximal digit / non-digit runs; digit runs of up to 18
// digits are numeric.
void tokenize(const uint8_t *name, size_t n, std::vector<Tok> &toks) {
    toks.clear();
    size_t i = 0;
    while (i < n) {
        const bool d = name[i] >= '0' && name[i] <= '9';
        const size_t s = i;
        while (i < n && (name[i] >= '0' && name[i] <= '9') == d) i++;
        Tok t{name + s, (uint32_t)(i - s), d && i - s <= kMaxNumDigits, 0};
        if (t.is_num)
            for (size_t k = s; k < i; k++) t.value = t.value * 10 + (name[k] - '0');
        toks.push_back(t);
    }
}

// Every role stream of one block, in payload order: counts, str_lens,
// str_data, num_vals, pads, op run counts / symbols / lengths, then the
// delta planes column by column.
struct BlockRoles {
    uint64_t n_records = 0;
    std::vector<uint8_t> raw;
    std::vector<uint64_t> len;  // stream lengths; streams lie back to back in raw
    uint8_t width[kCols] = {};
};

void build_roles(const uint8_t *names, const fqxv_rans_span *spans, uint64_t first, uint64_t count,
                 BlockRoles &B) {
    std::vector<uint8_t> counts, str_lens, str_data, num_vals, pads;
    std::vector<std::vector<uint8_t>> ops(kCols);
    std::vector<std::vector<uint64_t>> deltas(kCols);
    std::vector<Tok> prev, toks;
    for (uint64_t r = 0; r < count; r++) {
        const fqxv_rans_span &sp = spans[first + r];
        tokenize(names + sp.offset, sp.length, toks);
        for (size_t i = 0; i < toks.size(); i++) {
            const Tok &t = toks[i];
            const int col = (int)std::min<size_t>(i, kCols - 1);
            const Tok *p = i < prev.size() ? &prev[i] : nullptr;
            if (p && p->len == t.len && std::memcmp(p->p, t.p, t.len) == 0) {
                ops[col].push_back(kMatch);
            } else if (t.is_num) {
                // t.len - natural_digits(t.value): the leading zeros, all but a
                // last lone digit
                uint32_t lz = 0;
                while (lz + 1 < t.len && t.p[lz] == '0') lz++;
                const uint8_t pad = (uint8_t)lz;
                if (p && p->is_num) {
                    ops[col].push_back(kDelta);
                    deltas[col].push_back(zigzag((int64_t)((uint64_t)t.value - (uint64_t)p->value)));
                } else {
                    ops[col].push_back(kNum);
                    put_varint(num_vals, (uint64_t)t.value);
                }
                pads.push_back(pad);
            } else {
                ops[col].push_back(kStr);
                put_varint(str_lens, t.len);
                str_data.insert(str_data.end(), t.p, t.p + t.len);
            }
        }
        put_varint(counts, toks.size());
        std::swap(prev, toks);
    }
    B.n_records = count;
    auto add = [&](const std::vector<uint8_t> &s) {
        B.raw.insert(B.raw.end(), s.begin(), s.end());
        B.len.push_back(s.size());
    };
    add(counts);
    add(str_lens);
    add(str_data);
    add(num_vals);
    add(pads);
    // lib.rs:176-202: per column, runs as (symbol, varint length); the run
    // count of each column in its own stream
    std::vector<uint8_t> rc, rs, rl;
    for (const auto &col : ops) {
        uint64_t runs = 0;
        for (size_t i = 0; i < col.size();) {
            size_t r = 1;
            while (i + r < col.size() && col[i + r] == col[i]) r++;
            rs.push_back(col[i]);
            put_varint(rl, r);
            runs++;
            i += r;
        }
        put_varint(rc, runs);
    }
    add(rc);
    add(rs);
    add(rl);
    // lib.rs:118-137: each column's values as little-endian byte planes, as
    // many as the largest value needs (0: empty column)
    for (int c = 0; c < kCols; c++) {
        const auto &v = deltas[c];
        if (v.empty()) continue;
        const uint64_t m = *std::max_element(v.begin(), v.end());
        int w = 1;
        while (w < 8 && (m >> (8 * w))) w++;
        B.width[c] = (uint8_t)w;
        for (int p = 0; p < w; p++) {
            const size_t o = B.raw.size();
            B.raw.resize(o + v.size());
            for (size_t i = 0; i < v.size(); i++) B.raw[o + i] = (uint8_t)(v[i] >> (8 * p));
            B.len.push_back(v.size());
        }
    }
}

// ---- decode (lib.rs:543-650) ----------------------------------------------------

struct Reader {  // fqxv-bytes Reader with the tokenizer's errors (lib.rs:700-711)
    const uint8_t *p;
    uint64_t n, pos = 0;
    int u8(uint8_t &v) {
        if (pos >= n) return FQXV_TOK_E_TRUNCATED;
        v = p[pos++];
        return FQXV_RANS_OK;
    }
    int varint(uint64_t &v) {  // fqxv-bytes lib.rs:32-47: every failure is bad_varint
        v = 0;
        for (uint32_t shift = 0;;) {
            if (pos >= n) return FQXV_TOK_E_VARINT;
            const uint8_t b = p[pos++];
            v |= shift < 64 ? (uint64_t)(b & 0x7F) << shift : 0;
            if (!(b & 0x80)) return FQXV_RANS_OK;
            shift += 7;
            if (shift >= 64) return FQXV_TOK_E_VARINT;
        }
    }
    int take(uint64_t len, uint64_t &off) {
        if (len > n - pos) return FQXV_TOK_E_TRUNCATED;
        off = pos;
        pos += len;
        return FQXV_RANS_OK;
    }
};

// One payload's framing, read without decoding anything: the eight flat /
// op-run streams and the delta planes, with the first framing error and where
// it falls (the reference would meet it after everything framed before it).
struct Frame {
    int pre_err = FQXV_RANS_OK;  // version or record-count varint failure
    uint64_t n_records = 0;
    uint64_t max_out = 0;
    int nflat = 0;               // flat / op streams framed (of 8)
    uint64_t flat_off[kFlat] = {}, flat_len[kFlat] = {};
    // column c: its width was read when c < ncols_read; planes [plane_first[c],
    // plane_first[c] + planes_framed[c]) framed of width[c]
    int ncols_read = 0;
    uint64_t width[kCols] = {};
    uint32_t plane_first[kCols] = {}, planes_framed[kCols] = {};
    std::vector<uint64_t> plane_off, plane_len;
    int frame_err = FQXV_RANS_OK;  // the error that stopped the framing
};

void frame_payload(const uint8_t *src, uint64_t len, Frame &F) {
    Reader r{src, len};
    uint8_t v = 0;
    int e = r.u8(v);
    if (e == FQXV_RANS_OK && v != kVersion) e = FQXV_TOK_E_VERSION;
    if (e == FQXV_RANS_OK) e = r.varint(F.n_records);
    if (e) {
        F.pre_err = e;
        return;
    }
    F.max_out = len > (~0ull) / kMaxExpansion ? ~0ull : std::max(len * kMaxExpansion, kMinStreamBound);
    for (; F.nflat < kFlat; F.nflat++) {
        uint64_t l = 0, o = 0;
        if ((e = r.varint(l)) || (e = r.take(l, o))) {
            F.frame_err = e;
            return;
        }
        F.flat_off[F.nflat] = o;
        F.flat_len[F.nflat] = l;
    }
    for (; F.ncols_read < kCols; F.ncols_read++) {
        const int c = F.ncols_read;
        uint64_t w = 0;
        if ((e = r.varint(w))) {
            F.frame_err = e;
            return;
        }
        F.width[c] = w;
        F.plane_first[c] = (uint32_t)F.plane_off.size();
        for (uint64_t p = 0; p < w; p++) {
            uint64_t l = 0, o = 0;
            if ((e = r.varint(l)) || (e = r.take(l, o))) {
                F.ncols_read = c + 1;  // this column's width was read
                F.frame_err = e;
                return;
            }
            F.plane_off.push_back(o);
            F.plane_len.push_back(l);
            F.planes_framed[c]++;
        }
    }
}

uint64_t declared_len(const uint8_t *s, uint64_t len, bool *ok) {
    *ok = len >= 9;
    uint64_t n = 0;
    if (*ok)
        for (int k = 0; k < 8; k++) n |= (uint64_t)s[1 + k] << (8 * k);
    return n;
}

// A batch of streams to decode: spans into the payload arena, output
// capacities (their declared lengths), and for each stream the bound its
// decode_bounded call checks first.
struct DecodeList {
    std::vector<fqxv_rans_span> in, out;
    std::vector<int32_t> status;     // per stream: OK, the bound error, or the GPU's status
    std::vector<uint64_t> lens;
    std::vector<size_t> gpu_index;   // position in the GPU batch, or ~0 (bound error, no decode)
    uint64_t out_total = 0;
    size_t add(const uint8_t *arena, uint64_t off, uint64_t len, uint64_t bound) {
        const size_t k = status.size();
        bool ok;
        const uint64_t n = declared_len(arena + off, len, &ok);
        if (ok && n > bound) {  // lib.rs:226-231: checked before any decoding
            status.push_back(FQXV_RANS_E_BOUND);
            gpu_index.push_back(~(size_t)0);
            lens.push_back(0);
            return k;
        }
        status.push_back(FQXV_RANS_OK);
        lens.push_back(0);
        gpu_index.push_back(in.size());
        in.push_back(fqxv_rans_span{off, len});
        out.push_back(fqxv_rans_span{out_total, ok ? n : 0});
        out_total += ok ? n : 0;
        return k;
    }
    // Decodes the listed streams in one GPU pass; `dst` receives the outputs.
    int run(fqxv_rans_ctx *ctx, const uint8_t *arena, std::vector<uint8_t> &dst) {
        if (in.empty()) return FQXV_RANS_OK;
        dst.resize(std::max<uint64_t>(out_total, 1));
        std::vector<uint64_t> ol(in.size());
        std::vector<int32_t> st(in.size());
        const int r = fqxv_rans_decode_batch_host(ctx, arena, in.data(), in.size(), ~0ull, dst.data(), out.data(),
                                                  ol.data(), st.data());
        if (r != FQXV_RANS_OK && !(r >= FQXV_RANS_E_TRUNCATED && r <= FQXV_RANS_E_TRUNCATED_RENORM)) return r;
        for (size_t k = 0; k < status.size(); k++) {
            if (gpu_index[k] == ~(size_t)0) continue;
            status[k] = st[gpu_index[k]];
            lens[k] = ol[gpu_index[k]];
        }
        return FQXV_RANS_OK;
    }
    const uint8_t *data(const std::vector<uint8_t> &dst, size_t k) const { return dst.data() + out[gpu_index[k]].offset; }
};

struct BlockOut {
    int status = FQXV_RANS_OK;
    std::vector<uint8_t> bytes;
    std::vector<uint64_t> name_len;
};

// A rebuilt token: its bytes are in the block's output at [off, off + len).
struct OTok {
    uint64_t off;
    uint32_t len;
    bool is_num;
    int64_t value;
};

// The block's output bytes: written through a pointer, grown geometrically.
struct OutBuf {
    std::vector<uint8_t> &v;
    size_t n = 0;
    uint8_t *at(size_t need) {  // room for `need` more bytes at the end
        if (n + need > v.size()) v.resize(std::max<size_t>(2 * v.size(), n + need + 4096));
        return v.data() + n;
    }
};

// lib.rs:684-699 num_tok with the width lib.rs:620-634 gives it: the decimal
// value, zero-padded on the left to natural_digits(value) + pad, appended;
// returns its length. The digits are generated once and give the natural
// width too.
size_t put_num(OutBuf &ob, int64_t value, size_t pad) {
    char buf[24];
    int n = 0;
    uint64_t m = value < 0 ? 0 - (uint64_t)value : (uint64_t)value;
    do {
        buf[n++] = (char)('0' + m % 10);
        m /= 10;
    } while (m);
    const size_t natural = value > 0 ? (size_t)n : 1;  // lib.rs:256-265
    if (value < 0) buf[n++] = '-';
    const size_t len = std::max<size_t>(natural + pad, (size_t)n);
    uint8_t *w = ob.at(len);
    size_t k = 0;
    for (; k + n < len; k++) w[k] = '0';
    while (n) w[k++] = (uint8_t)buf[--n];
    ob.n += len;
    return len;
}

// lib.rs:580-650: names from the decoded role streams, written straight into
// the block's output (a MATCH copies the previous name's token).
int rebuild_names(uint64_t n_records, const uint8_t *counts, uint64_t ncounts, const uint8_t *str_lens,
                  uint64_t nsl, const uint8_t *str_data, uint64_t nsd, const uint8_t *num_vals, uint64_t nnv,
                  const uint8_t *pads, uint64_t npads, const std::vector<std::vector<uint8_t>> &ops,
                  const std::vector<std::vector<uint64_t>> &deltas, BlockOut &out) {
    Reader op[kCols];
    for (int c = 0; c < kCols; c++) op[c] = Reader{ops[c].data(), ops[c].size()};
    size_t dpos[kCols] = {};
    Reader cc{counts, ncounts}, cl{str_lens, nsl}, cn{num_vals, nnv};
    uint64_t str_pos = 0, pad_pos = 0;
    std::vector<OTok> prev, cur;
    prev.reserve(64);
    cur.reserve(64);
    OutBuf ob{out.bytes};
    out.bytes.resize(nsd + 48 * std::min<uint64_t>(n_records, 1u << 20) + 4096);
    out.name_len.reserve(n_records);
    int e;
    for (uint64_t rec = 0; rec < n_records; rec++) {
        uint64_t nt = 0;
        if ((e = cc.varint(nt))) return e;
        cur.clear();
        const size_t name_start = ob.n;
        for (uint64_t t = 0; t < nt; t++) {
            const size_t col = std::min<size_t>(cur.size(), kCols - 1);
            uint8_t o = 0;
            if ((e = op[col].u8(o))) return e;
            const size_t at = ob.n;
            if (o == kMatch) {
                if (cur.size() >= prev.size()) return FQXV_TOK_E_MATCH;
                const OTok p = prev[cur.size()];
                uint8_t *w = ob.at(p.len);
                std::memcpy(w, ob.v.data() + p.off, p.len);
                ob.n += p.len;
                cur.push_back(OTok{at, p.len, p.is_num, p.value});
            } else if (o == kStr) {
                uint64_t l = 0;
                if ((e = cl.varint(l))) return e;
                if (l > nsd || str_pos > nsd - l) return FQXV_TOK_E_STR_UNDERRUN;
                std::memcpy(ob.at(l), str_data + str_pos, l);
                ob.n += l;
                str_pos += l;
                cur.push_back(OTok{at, (uint32_t)l, false, 0});
            } else if (o == kNum || o == kDelta) {
                int64_t value;
                if (o == kNum) {
                    uint64_t v = 0;
                    if ((e = cn.varint(v))) return e;
                    value = (int64_t)v;
                } else {
                    if (dpos[col] >= deltas[col].size()) return FQXV_TOK_E_DELTA_UNDERRUN;
                    const int64_t d = unzigzag(deltas[col][dpos[col]++]);
                    if (cur.size() >= prev.size() || !prev[cur.size()].is_num) return FQXV_TOK_E_DELTA_PRIOR;
                    value = (int64_t)((uint64_t)prev[cur.size()].value + (uint64_t)d);
                }
                if (pad_pos >= npads) return FQXV_TOK_E_PAD_UNDERRUN;
                const size_t len = put_num(ob, value, pads[pad_pos++]);
                cur.push_back(OTok{at, (uint32_t)len, true, value});
            } else {
                return FQXV_TOK_E_UNKNOWN_OP;
            }
        }
        out.name_len.push_back(ob.n - name_start);
        std::swap(prev, cur);
    }
    out.bytes.resize(ob.n);
    return FQXV_RANS_OK;
}

}  // namespace

extern "C" {

int fqxv_tok_encode_host(fqxv_rans_ctx *ctx, const uint8_t *h_names, const fqxv_rans_span *name_spans,
                         size_t nnames, const fqxv_rans_span *blocks, size_t nblocks, uint8_t *h_dst,
                         uint64_t cap, fqxv_rans_span *out, uint64_t *needed) {
    if (!ctx || (nblocks && (!blocks || !out)) || (nnames && (!name_spans || !h_names))) return FQXV_RANS_E_INVALID_ARG;
    for (size_t b = 0; b < nblocks; b++)
        if (blocks[b].offset > nnames || blocks[b].length > nnames - blocks[b].offset) return FQXV_RANS_E_INVALID_ARG;
    std::vector<BlockRoles> roles(nblocks);
    parallel_for(nblocks, [&](size_t b) {
        build_roles(h_names, name_spans, blocks[b].offset, blocks[b].length, roles[b]);
    });
    // every role stream of every block in one arena, coded in one pass
    size_t ns = 0;
    uint64_t raw_total = 0;
    for (auto &B : roles) {
        ns += B.len.size();
        raw_total += B.raw.size();
    }
    std::vector<uint8_t> arena(std::max<uint64_t>(raw_total, 1));
    std::vector<fqxv_rans_span> sp(ns), coded(ns);
    uint64_t pos = 0, code_cap = 0;
    size_t k = 0;
    for (auto &B : roles) {
        if (!B.raw.empty()) std::memcpy(arena.data() + pos, B.raw.data(), B.raw.size());
        uint64_t o = pos;
        for (uint64_t l : B.len) {
            sp[k++] = fqxv_rans_span{o, l};
            o += l;
            code_cap += 9 + 512 + 128 + 2 * l;  // the order-0 bound covers the smaller of the two
        }
        pos += B.raw.size();
    }
    std::vector<uint8_t> cbuf(std::max<uint64_t>(code_cap, 1));
    if (ns) {
        const int st = fqxv_rans_encode_batch_host(ctx, arena.data(), sp.data(), ns, FQXV_RANS_BEST_TIE0,
                                                   cbuf.data(), code_cap, coded.data(), nullptr);
        if (st) return st;
    }
    // payloads: [1][varint n][8 x (varint len, stream)][64 x (varint width, planes)]
    std::vector<uint64_t> psize(nblocks);
    std::vector<size_t> first(nblocks + 1, 0);
    for (size_t b = 0; b < nblocks; b++) first[b + 1] = first[b] + roles[b].len.size();
    auto vlen = [](uint64_t v) {
        uint64_t n = 1;
        while (v >>= 7) n++;
        return n;
    };
    uint64_t total = 0;
    for (size_t b = 0; b < nblocks; b++) {
        uint64_t t = 1 + vlen(roles[b].n_records);
        for (size_t s = first[b]; s < first[b + 1]; s++) t += vlen(coded[s].length) + coded[s].length;
        for (int c = 0; c < kCols; c++) t += vlen(roles[b].width[c]);
        psize[b] = t;
        total += t;
    }
    if (needed) *needed = total;
    if (total > cap || (total && !h_dst)) return FQXV_RANS_E_DST_TOO_SMALL;
    std::vector<uint64_t> start(nblocks);
    for (size_t b = 0, o = 0; b < nblocks; b++) {
        start[b] = o;
        o += psize[b];
    }
    parallel_for(nblocks, [&](size_t b) {
        std::vector<uint8_t> p;
        p.reserve(psize[b]);
        p.push_back(kVersion);
        put_varint(p, roles[b].n_records);
        auto stream = [&](size_t s) {
            put_varint(p, coded[s].length);
            p.insert(p.end(), cbuf.data() + coded[s].offset, cbuf.data() + coded[s].offset + coded[s].length);
        };
        size_t s = first[b];
        for (int f = 0; f < kFlat; f++) stream(s++);
        for (int c = 0; c < kCols; c++) {
            put_varint(p, roles[b].width[c]);
            for (int q = 0; q < roles[b].width[c]; q++) stream(s++);
        }
        std::memcpy(h_dst + start[b], p.data(), p.size());
        out[b] = fqxv_rans_span{start[b], p.size()};
    });
    return FQXV_RANS_OK;
}

int fqxv_tok_decode_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, const fqxv_rans_span *payloads, size_t nblocks,
                         uint8_t *h_names, uint64_t names_cap, fqxv_rans_span *name_spans, uint64_t spans_cap,
                         fqxv_rans_span *blocks, int32_t *status, uint64_t *names_needed, uint64_t *spans_needed) {
    if (!ctx || (nblocks && (!payloads || !h_src || !blocks || !status))) return FQXV_RANS_E_INVALID_ARG;
    std::vector<Frame> F(nblocks);
    parallel_for(nblocks, [&](size_t b) { frame_payload(h_src + payloads[b].offset, payloads[b].length, F[b]); });
    std::vector<BlockOut> out(nblocks);
    // pass 1: the flat and op-run streams (decode_bounded by max_out, lib.rs:107-110)
    DecodeList d1;
    std::vector<size_t> flat_first(nblocks);
    for (size_t b = 0; b < nblocks; b++) {
        flat_first[b] = d1.status.size();
        for (int f = 0; f < F[b].nflat; f++)
            d1.add(h_src, payloads[b].offset + F[b].flat_off[f], F[b].flat_len[f], F[b].max_out);
    }
    std::vector<uint8_t> dst1;
    int r = d1.run(ctx, h_src, dst1);
    if (r) return r;
    // Walk each block in the reference's order up to its planes: the first
    // error met (a framing error after every stream framed before it, a
    // stream's decode error, or a content check) is the block's status.
    std::vector<std::vector<std::vector<uint8_t>>> ops(nblocks);
    std::vector<std::vector<uint64_t>> n_delta(nblocks);
    parallel_for(nblocks, [&](size_t b) {
        Frame &f = F[b];
        BlockOut &o = out[b];
        if (f.pre_err) {
            o.status = f.pre_err;
            return;
        }
        for (int s = 0; s < kFlat; s++) {
            if (s >= f.nflat) {
                o.status = f.frame_err;
                return;
            }
            const size_t k = flat_first[b] + s;
            if (d1.status[k]) {
                o.status = d1.status[k];
                return;
            }
            if (s == 0 && f.n_records > d1.lens[k]) {  // lib.rs:564-566
                o.status = FQXV_TOK_E_RECORDS;
                return;
            }
        }
        // lib.rs:205-254: the op columns from their runs
        const size_t k0 = flat_first[b] + 5;
        Reader rc{d1.lens[k0] ? d1.data(dst1, k0) : nullptr, d1.lens[k0]};
        const uint8_t *syms = d1.lens[k0 + 1] ? d1.data(dst1, k0 + 1) : nullptr;
        const uint64_t nsyms = d1.lens[k0 + 1];
        Reader rl{d1.lens[k0 + 2] ? d1.data(dst1, k0 + 2) : nullptr, d1.lens[k0 + 2]};
        uint64_t sym_pos = 0, total_ops = 0;
        ops[b].assign(kCols, {});
        for (int c = 0; c < kCols; c++) {
            uint64_t n_runs = 0;
            int e = rc.varint(n_runs);
            if (e) {
                o.status = e;
                return;
            }
            auto &col = ops[b][c];
            for (uint64_t q = 0; q < n_runs; q++) {
                if (sym_pos >= nsyms) {
                    o.status = FQXV_TOK_E_SYM_UNDERRUN;
                    return;
                }
                const uint8_t s = syms[sym_pos++];
                uint64_t run = 0;
                if ((e = rl.varint(run))) {
                    o.status = e;
                    return;
                }
                if (run > f.n_records || col.size() > f.n_records - run) {
                    o.status = FQXV_TOK_E_RUN_TOO_LONG;
                    return;
                }
                if (run > f.max_out || total_ops > f.max_out - run) {
                    o.status = FQXV_TOK_E_OPS_BOUND;
                    return;
                }
                total_ops += run;
                col.insert(col.end(), run, s);
            }
        }
        n_delta[b].assign(kCols, 0);
        for (int c = 0; c < kCols; c++)
            n_delta[b][c] = (uint64_t)std::count(ops[b][c].begin(), ops[b][c].end(), kDelta);
    });
    // pass 2: the delta planes (decode_bounded by the column's delta count,
    // lib.rs:140-170)
    DecodeList d2;
    std::vector<size_t> plane_first(nblocks);
    for (size_t b = 0; b < nblocks; b++) {
        plane_first[b] = d2.status.size();
        if (out[b].status) continue;
        const Frame &f = F[b];
        for (int c = 0; c < f.ncols_read; c++)
            for (uint32_t q = 0; q < f.planes_framed[c]; q++) {
                const size_t i = f.plane_first[c] + q;
                d2.add(h_src, payloads[b].offset + f.plane_off[i], f.plane_len[i], n_delta[b][c]);
            }
    }
    std::vector<uint8_t> dst2;
    r = d2.run(ctx, h_src, dst2);
    if (r) return r;
    parallel_for(nblocks, [&](size_t b) {
        BlockOut &o = out[b];
        if (o.status) return;
        const Frame &f = F[b];
        std::vector<std::vector<uint64_t>> deltas(kCols);
        size_t k = plane_first[b];
        for (int c = 0; c < kCols; c++) {
            if (c >= f.ncols_read) {
                o.status = f.frame_err;
                return;
            }
            if (f.width[c] == 0) continue;
            const uint64_t n = n_delta[b][c];
            auto &vals = deltas[c];
            vals.assign(n, 0);
            for (uint64_t q = 0; q < f.width[c]; q++) {
                if (q >= f.planes_framed[c]) {
                    o.status = f.frame_err;
                    return;
                }
                if (d2.status[k]) {
                    o.status = d2.status[k];
                    return;
                }
                if (d2.lens[k] != n) {
                    o.status = FQXV_TOK_E_PLANE_LEN;
                    return;
                }
                const uint8_t *pl = n ? d2.data(dst2, k) : nullptr;
                for (uint64_t i = 0; i < n; i++) vals[i] |= (uint64_t)pl[i] << (8 * q);
                k++;
            }
        }
        const size_t f0 = flat_first[b];
        auto ptr = [&](int s) -> const uint8_t * { return d1.lens[f0 + s] ? d1.data(dst1, f0 + s) : nullptr; };
        o.status = rebuild_names(f.n_records, ptr(0), d1.lens[f0], ptr(1), d1.lens[f0 + 1], ptr(2),
                                 d1.lens[f0 + 2], ptr(3), d1.lens[f0 + 3], ptr(4), d1.lens[f0 + 4], ops[b], deltas,
                                 o);
        if (o.status) {
            o.bytes.clear();
            o.name_len.clear();
        }
    });
    uint64_t nb_bytes = 0, nb_names = 0;
    for (auto &o : out) {
        nb_bytes += o.bytes.size();
        nb_names += o.name_len.size();
    }
    if (names_needed) *names_needed = nb_bytes;
    if (spans_needed) *spans_needed = nb_names;
    if (nb_bytes > names_cap || nb_names > spans_cap || (nb_bytes && !h_names) || (nb_names && !name_spans))
        return FQXV_RANS_E_DST_TOO_SMALL;
    int first = FQXV_RANS_OK;
    uint64_t bo = 0, no = 0;
    for (size_t b = 0; b < nblocks; b++) {
        const BlockOut &o = out[b];
        status[b] = o.status;
        if (o.status && first == FQXV_RANS_OK) first = o.status;
        blocks[b] = fqxv_rans_span{no, o.name_len.size()};
        if (!o.bytes.empty()) std::memcpy(h_names + bo, o.bytes.data(), o.bytes.size());
        for (uint64_t l : o.name_len) {
            name_spans[no++] = fqxv_rans_span{bo, l};
            bo += l;
        }
    }
    return first;
}

}  // extern "C"
