// put_stream / get_stream of crates/fqxv-lroverlap/src/codec.rs:289-363,
// batched over the GPU coder (include/fqxv_streams_gpu.h). Framing is host
// C++; every stream of a call is coded or decoded in one batch pass.
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "../../include/fqxv_streams_gpu.h"

namespace {

uint64_t varint_len(uint64_t v) {
    uint64_t n = 1;
    while (v >>= 7) n++;
    return n;
}

uint8_t *put_varint(uint8_t *p, uint64_t v) {  // fqxv-bytes lib.rs:14-24
    for (;;) {
        const uint8_t b = (uint8_t)(v & 0x7F);
        v >>= 7;
        if (!v) {
            *p++ = b;
            return p;
        }
        *p++ = b | 0x80;
    }
}

// fqxv-bytes lib.rs:32-47: None on truncation or more than 64 bits.
bool read_varint(const uint8_t *s, uint64_t len, uint64_t &pos, uint64_t &v) {
    v = 0;
    for (uint32_t shift = 0;;) {
        if (pos >= len) return false;
        const uint8_t b = s[pos++];
        v |= (uint64_t)(b & 0x7F) << shift;
        if (!(b & 0x80)) return true;
        shift += 7;
        if (shift >= 64) return false;
    }
}

}  // namespace

extern "C" {

int fqxv_put_streams_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, const fqxv_rans_span *raw, size_t n,
                          uint8_t *h_dst, uint64_t cap, fqxv_rans_span *out, uint64_t *needed) {
    if (!ctx || (n && (!raw || !out))) return FQXV_RANS_E_INVALID_ARG;
    // the non-empty streams, coded at both orders, the smaller kept, ties to
    // order-1 (codec.rs:297-299)
    std::vector<fqxv_rans_span> sp, coded;
    std::vector<size_t> idx;
    uint64_t code_cap = 0;
    for (size_t i = 0; i < n; i++)
        if (raw[i].length) {
            if (!h_src) return FQXV_RANS_E_INVALID_ARG;
            idx.push_back(i);
            sp.push_back(raw[i]);
            code_cap += 9 + 512 + 128 + 2 * raw[i].length;
        }
    coded.resize(sp.size());
    std::unique_ptr<uint8_t[]> cbuf(new uint8_t[std::max<uint64_t>(code_cap, 1)]);
    if (!sp.empty()) {
        const int st = fqxv_rans_encode_batch_host(ctx, h_src, sp.data(), sp.size(), FQXV_RANS_BEST_TIE1,
                                                   cbuf.get(), code_cap, coded.data(), nullptr);
        if (st) return st;
    }
    uint64_t total = 0;
    size_t k = 0;
    std::vector<uint64_t> flen(n);
    for (size_t i = 0; i < n; i++) {
        flen[i] = varint_len(raw[i].length);
        if (raw[i].length) {
            flen[i] += varint_len(coded[k].length) + coded[k].length;
            k++;
        }
        total += flen[i];
    }
    if (needed) *needed = total;
    if (total > cap || (total && !h_dst)) return FQXV_RANS_E_DST_TOO_SMALL;
    uint64_t pos = 0;
    k = 0;
    for (size_t i = 0; i < n; i++) {
        uint8_t *p = put_varint(h_dst + pos, raw[i].length);
        if (raw[i].length) {
            p = put_varint(p, coded[k].length);
            std::memcpy(p, cbuf.get() + coded[k].offset, coded[k].length);
            k++;
        }
        out[i] = fqxv_rans_span{pos, flen[i]};
        pos += flen[i];
    }
    return FQXV_RANS_OK;
}

int fqxv_get_streams_host(fqxv_rans_ctx *ctx, const uint8_t *h_src, uint64_t len, uint64_t pos, size_t n,
                          uint8_t *h_dst, uint64_t cap, fqxv_rans_span *out, int32_t *status, uint64_t *end_pos,
                          uint64_t *needed) {
    if (!ctx || (n && (!out || !status)) || (len && !h_src) || pos > len) return FQXV_RANS_E_INVALID_ARG;
    // framing (codec.rs:349-357); a frame that fails ends the walk
    struct Fr {
        uint64_t raw_len, off, enc_len;
        bool ok;
    };
    std::vector<Fr> fr(n, Fr{0, 0, 0, false});
    size_t nread = 0;
    for (; nread < n; nread++) {
        Fr &f = fr[nread];
        if (!read_varint(h_src, len, pos, f.raw_len)) break;
        if (f.raw_len == 0) {
            f.ok = true;
            continue;
        }
        if (!read_varint(h_src, len, pos, f.enc_len) || f.enc_len > len - pos) break;
        f.off = pos;
        pos += f.enc_len;
        f.ok = true;
    }
    if (end_pos) *end_pos = pos;
    // decode_bounded(enc, raw_len): the declared length is checked first; a
    // stream that cannot hold raw_len bytes fails before any output is sized
    std::vector<fqxv_rans_span> in, osp;
    std::vector<size_t> idx;
    std::vector<int32_t> st(n, FQXV_STREAM_E_CORRUPT);
    uint64_t total = 0;
    for (size_t i = 0; i < nread; i++) {
        const Fr &f = fr[i];
        if (f.raw_len == 0) {
            st[i] = FQXV_RANS_OK;
            continue;
        }
        uint64_t declared = ~0ull;
        if (f.enc_len >= 9) {
            declared = 0;
            for (int b = 0; b < 8; b++) declared |= (uint64_t)h_src[f.off + 1 + b] << (8 * b);
        }
        if (f.enc_len >= 9 && declared != f.raw_len) continue;  // over the bound, or a length mismatch
        idx.push_back(i);
        in.push_back(fqxv_rans_span{f.off, f.enc_len});
        osp.push_back(fqxv_rans_span{total, f.enc_len >= 9 ? f.raw_len : 0});
        total += f.enc_len >= 9 ? f.raw_len : 0;
    }
    if (needed) *needed = total;
    if (total > cap || (total && !h_dst)) return FQXV_RANS_E_DST_TOO_SMALL;
    if (!in.empty()) {
        std::vector<uint64_t> ol(in.size());
        std::vector<int32_t> ds(in.size());
        const int r = fqxv_rans_decode_batch_host(ctx, h_src, in.data(), in.size(), ~0ull, h_dst, osp.data(),
                                                  ol.data(), ds.data());
        if (r != FQXV_RANS_OK && !(r >= FQXV_RANS_E_TRUNCATED && r <= FQXV_RANS_E_TRUNCATED_RENORM)) return r;
        for (size_t j = 0; j < in.size(); j++)
            if (ds[j] == FQXV_RANS_OK && ol[j] == fr[idx[j]].raw_len) st[idx[j]] = FQXV_RANS_OK;
    }
    // the reference stops at the first failure: later frames are not read
    int first = FQXV_RANS_OK;
    uint64_t o = 0;
    for (size_t i = 0; i < n; i++) {
        if (first != FQXV_RANS_OK) st[i] = FQXV_STREAM_E_CORRUPT;
        status[i] = st[i];
        if (st[i] != FQXV_RANS_OK && first == FQXV_RANS_OK) first = st[i];
        const uint64_t l = st[i] == FQXV_RANS_OK ? fr[i].raw_len : 0;
        out[i] = fqxv_rans_span{o, l};
        o += l;
    }
    // every stream before the first failure decoded in place at its packed
    // offset; the outputs of streams after it are simply not reported
    return first;
}

}  // extern "C"
