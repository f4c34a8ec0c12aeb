"""Batched device API parity: many blocks per pass, against the oracle block
by block; batched and plain per-block forms give the same bytes; full-size
workloads checked through round trips and against the oracle."""

import numpy as np
import pytest

from fqxv_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def codec():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from fqxv_b200.batch import Codec

    c = Codec(0)
    yield c
    c.close()


def _dev(a):
    import torch

    return torch.from_numpy(np.array(a, dtype=np.uint8, copy=True)).to("cuda")


def _oracle_best(orc, blk, tie_to_one=False):
    e0, e1 = orc.encode(blk, 0), orc.encode(blk, 1)
    if tie_to_one:
        return e1 if len(e1) <= len(e0) else e0
    return e1 if len(e1) < len(e0) else e0


def _roundtrip_check(codec, data, spans, d_out, out_spans):
    import torch

    dsp = out_spans.copy()
    dst = np.zeros_like(spans)
    dst[:, 0] = spans[:, 0]
    dst[:, 1] = spans[:, 1]
    d_dec, lens, st = codec.decode_batch(d_out, dsp, dst)
    assert (st == 0).all()
    assert (lens == spans[:, 1]).all()
    torch.cuda.synchronize()
    assert np.array_equal(d_dec[:len(data)].cpu().numpy(), data)


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_mixed_batch_matches_oracle(codec, orc, mode):
    data, spans, kinds = W.config2(nblocks=48, lo=1, hi=300_000, seed=100 + mode)
    d_src = _dev(data)
    d_out, out_spans, orders = codec.encode_batch(d_src, spans, mode)
    out = d_out.cpu().numpy()
    pos = 0
    for i, (off, ln) in enumerate(spans):
        blk = data[int(off):int(off + ln)].tobytes()
        if mode in (0, 1):
            ref = orc.encode(blk, mode)
        else:
            ref = _oracle_best(orc, blk, tie_to_one=(mode == 3))
        o, l = int(out_spans[i, 0]), int(out_spans[i, 1])
        assert o == pos, "streams are back to back in block order"
        assert out[o:o + l].tobytes() == ref, (i, kinds[i], len(blk))
        assert orders[i] == ref[0]
        pos += l
    _roundtrip_check(codec, data, spans, d_out, out_spans)


@pytest.mark.parametrize("mode", [1, 2])
def test_keyless_order1_encode_matches_oracle(codec, orc, mode):
    """Order-1 encode without the per-position key array (enc_o1_keys = 0):
    the same bytes as the oracle, small and odd block lengths included."""
    data, spans, kinds = W.config2(nblocks=48, lo=1, hi=300_000, seed=300 + mode)
    extra = [np.random.default_rng(s).integers(0, 256, s, dtype=np.uint8) for s in (1, 2, 31, 32, 33, 511, 512, 513, 1025)]
    data = np.concatenate([data] + extra)
    lens = [int(x) for x in spans[:, 1]] + [len(e) for e in extra]
    offs = np.concatenate([[0], np.cumsum(lens)[:-1]])
    spans = np.stack([offs, lens], 1).astype(np.uint64)
    old = codec.get_param("enc_o1_keys")
    codec.set_param("enc_o1_keys", 0)
    try:
        d_out, out_spans, orders = codec.encode_batch(_dev(data), spans, mode)
    finally:
        codec.set_param("enc_o1_keys", old)
    out = d_out.cpu().numpy()
    ref, roff, rlen = orc.encode_batch(data, spans[:, 0], spans[:, 1], mode)
    for i in range(len(spans)):
        got = out[int(out_spans[i, 0]):int(out_spans[i, 0] + out_spans[i, 1])]
        assert np.array_equal(got, ref[int(roff[i]):int(roff[i] + rlen[i])]), (i, lens[i])
    _roundtrip_check(codec, data, spans, d_out, out_spans)


def test_plain_form_equals_batched(codec):
    data, spans, _ = W.config2(nblocks=24, lo=100, hi=200_000, seed=7)
    d_src = _dev(data)
    for mode in (0, 1, 2):
        a, sa, oa = codec.encode_batch(d_src, spans, mode, persistent=True)
        b, sb, ob = codec.encode_batch(d_src, spans, mode, persistent=False)
        assert np.array_equal(sa, sb) and np.array_equal(oa, ob)
        n = int(sa[-1, 0] + sa[-1, 1])
        assert np.array_equal(a[:n].cpu().numpy(), b[:n].cpu().numpy())
        dst = spans.copy()
        d1, l1, s1 = codec.decode_batch(a, sa, dst, persistent=True)
        d2, l2, s2 = codec.decode_batch(a, sa, dst, persistent=False)
        assert (s1 == 0).all() and (s2 == 0).all()
        assert np.array_equal(d1[:len(data)].cpu().numpy(), d2[:len(data)].cpu().numpy())


def test_config0_binned_order0_full_size(codec, orc):
    data, spans = W.config0()
    d_out, sp, _ = codec.encode_batch(_dev(data), spans, 0)
    ref = orc.encode(data.tobytes(), 0)
    assert d_out[:int(sp[0, 1])].cpu().numpy().tobytes() == ref
    _roundtrip_check(codec, data, spans, d_out, sp)


def test_config1_full_quality_order1_full_size(codec, orc):
    data, spans = W.config1()
    d_out, sp, _ = codec.encode_batch(_dev(data), spans, 1)
    out = d_out.cpu().numpy()
    ref, roff, rlen = orc.encode_batch(data, spans[:, 0], spans[:, 1], 1)
    for i in range(len(spans)):
        got = out[int(sp[i, 0]):int(sp[i, 0] + sp[i, 1])]
        want = ref[int(roff[i]):int(roff[i] + rlen[i])]
        assert np.array_equal(got, want), i
    _roundtrip_check(codec, data, spans, d_out, sp)


def test_ont_blocks_cpu_encoded_gpu_decoded(codec, orc):
    data, spans = W.config3_ont(nreads=120, lo=64 << 10, hi=1 << 20, seed=3)
    enc, eoff, elen = orc.encode_batch(data, spans[:, 0], spans[:, 1], 1)
    cs = np.stack([eoff, elen], axis=1)
    d_dec, lens, st = codec.decode_batch(_dev(enc), cs, spans)
    assert (st == 0).all() and (lens == spans[:, 1]).all()
    assert np.array_equal(d_dec[:len(data)].cpu().numpy(), data)


def test_decode_batch_per_block_status(codec, orc):
    rng = np.random.default_rng(1)
    streams, want = [], []
    for i in range(40):
        blk = rng.integers(0, 30, int(rng.integers(0, 5000))).astype(np.uint8).tobytes()
        e = bytearray(orc.encode(blk, i % 2))
        if i % 3 == 0 and len(e) > 20:
            e = e[:int(rng.integers(9, len(e)))]
        if i % 5 == 0 and len(e) > 12:
            e[10] ^= 0x5A
        streams.append(bytes(e))
        want.append(orc.decode_status(bytes(e), max_len=1 << 16))
    lens = np.array([len(s) for s in streams], np.uint64)
    offs = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.uint64)
    arena = np.frombuffer(b"".join(streams), np.uint8)
    caps = np.full(40, 1 << 16, np.uint64)
    doffs = (np.arange(40, dtype=np.uint64) << np.uint64(16))
    d_dec, olens, st = codec.decode_batch(_dev(arena), np.stack([offs, lens], 1), np.stack([doffs, caps], 1),
                                          max_len=1 << 16, raise_on_error=False)
    dec = d_dec.cpu().numpy()
    for i, (ws, wb) in enumerate(want):
        assert st[i] == ws, i
        if ws == 0:
            assert dec[int(doffs[i]):int(doffs[i]) + int(olens[i])].tobytes() == wb


def test_host_decode_pinned_and_pageable_agree(codec, orc):
    """A pinned destination is written in place by the kernels, a pageable
    one through a staging copy; both give the oracle's bytes and statuses."""
    import torch

    rng = np.random.default_rng(9)
    streams, want = [], []
    for i in range(24):
        blk = W.GENERATORS[list(W.GENERATORS)[i % 4]](int(rng.integers(1, 200_000)), 40 + i).tobytes()
        e = bytearray(orc.encode(blk, i % 2))
        if i % 7 == 3:
            e = e[:len(e) // 2]      # truncated
        streams.append(bytes(e))
        want.append(orc.decode_status(bytes(e), max_len=1 << 18))
    lens = np.array([len(s) for s in streams], np.uint64)
    offs = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.uint64)
    arena = np.frombuffer(b"".join(streams), np.uint8)
    caps = np.full(len(streams), 1 << 18, np.uint64)
    doffs = np.arange(len(streams), dtype=np.uint64) << np.uint64(18)
    spans, ospans = np.stack([offs, lens], 1), np.stack([doffs, caps], 1)
    pin_src = torch.from_numpy(arena.copy()).pin_memory().numpy()
    pin_dst = torch.zeros(len(streams) << 18, dtype=torch.uint8).pin_memory().numpy()
    page_dst = np.zeros(len(streams) << 18, np.uint8)
    l1, s1 = codec.decode_batch_host(pin_src, spans, ospans, pin_dst, max_len=1 << 18, raise_on_error=False)
    l2, s2 = codec.decode_batch_host(arena.copy(), spans, ospans, page_dst, max_len=1 << 18, raise_on_error=False)
    for i, (ws, wb) in enumerate(want):
        assert s1[i] == ws and s2[i] == ws, i
        if ws == 0:
            o = int(doffs[i])
            assert pin_dst[o:o + int(l1[i])].tobytes() == wb
            assert page_dst[o:o + int(l2[i])].tobytes() == wb


def test_pinned_destination_mirror_unaligned(codec, orc):
    """A large pinned destination is filled by the decoding CTAs' copies of
    their streams (16-byte stores between ragged ends): a destination that
    starts at an odd address, streams back to back at odd offsets, lengths
    from 1 byte up, both orders and a truncated stream in the middle."""
    import torch

    rng = np.random.default_rng(19)
    blocks = [W.GENERATORS[list(W.GENERATORS)[i % 4]](n, 70 + i)
              for i, n in enumerate([1, 2, 15, 16, 17, 31, 33, 1000, 70_001, 300_000, 1 << 20, 2_500_001])]
    blocks += [W.GENERATORS["full"](int(rng.integers(1, 400_000)), 90 + i) for i in range(20)]
    streams = [orc.encode(b.tobytes(), i % 2) for i, b in enumerate(blocks)]
    streams[9] = streams[9][:len(streams[9]) // 3]
    lens = np.array([len(x) for x in streams], np.uint64)
    offs = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.uint64)
    nout = np.array([len(b) for b in blocks], np.uint64)
    doffs = np.concatenate([[0], np.cumsum(nout)[:-1]]).astype(np.uint64)
    total = int(nout.sum())
    assert total >= (4 << 20)
    h_in = torch.from_numpy(np.frombuffer(b"".join(streams), np.uint8).copy()).pin_memory().numpy()
    pinned = torch.zeros(total + 64, dtype=torch.uint8).pin_memory().numpy()
    h_dst = pinned[5:5 + total]
    l, st = codec.decode_batch_host(h_in, np.stack([offs, lens], 1), np.stack([doffs, nout], 1), h_dst,
                                    raise_on_error=False)
    for i, b in enumerate(blocks):
        ws, wb = orc.decode_status(streams[i])
        assert st[i] == ws, i
        if ws == 0:
            o = int(doffs[i])
            assert h_dst[o:o + int(l[i])].tobytes() == wb == b.tobytes(), i
    assert not pinned[:5].any() and not pinned[5 + total:].any()


def test_host_pipeline_settings_change_no_byte(codec):
    """The host-buffer pipeline choices (input read in place or copied, output
    mirrored by the decoding CTAs or copied after the batch, chunk counts)
    give the same streams and the same decoded bytes."""
    import torch

    data, spans, _ = W.config2(nblocks=700, lo=1000, hi=400_000, seed=55)
    assert len(data) >= (32 << 20)  # large enough to be cut into chunks
    h_src = torch.from_numpy(data.copy()).pin_memory().numpy()
    bound = codec.encode_bound(spans, 2)
    ref = None
    keys = ("host_enc_chunks", "host_dec_chunks", "host_in_place", "host_out_mirror")
    old = {k: codec.get_param(k) for k in keys}
    try:
        for enc_chunks, dec_chunks, in_place, mirror in ((1, 1, -1, 1), (4, 4, 0, 0), (2, 1, 1, 1), (8, 2, 1, 0)):
            codec.set_param("host_enc_chunks", enc_chunks)
            codec.set_param("host_dec_chunks", dec_chunks)
            codec.set_param("host_in_place", in_place)
            codec.set_param("host_out_mirror", mirror)
            h_enc = torch.zeros(bound, dtype=torch.uint8).pin_memory().numpy()
            es, _ = codec.encode_batch_host(h_src, spans, 2, h_enc)
            total = int(es[-1, 0] + es[-1, 1])
            if ref is None:
                ref = (es.copy(), h_enc[:total].copy())
            assert np.array_equal(es, ref[0]) and np.array_equal(h_enc[:total], ref[1])
            h_dec = torch.zeros(len(data), dtype=torch.uint8).pin_memory().numpy()
            lens, st = codec.decode_batch_host(h_enc, es, spans, h_dec)
            assert (st == 0).all() and np.array_equal(h_dec, data)
    finally:
        for k, v in old.items():
            codec.set_param(k, v)


def test_small_alphabet_order1_statuses_match_oracle(codec, orc):
    """Order-1 streams of small alphabets (the one-warp decoder): good,
    truncated and corrupted streams give the oracle's bytes and statuses."""
    rng = np.random.default_rng(21)
    streams, want = [], []
    for i in range(60):
        k = int(rng.integers(1, 9))
        blk = rng.integers(0, k, int(rng.integers(1, 40_000))).astype(np.uint8)
        blk = (blk + 60).tobytes()
        e = bytearray(orc.encode(blk, 1))
        if i % 4 == 1:
            e = e[:int(rng.integers(9, len(e)))]
        elif i % 4 == 2 and len(e) > 200:
            for _ in range(3):
                e[int(rng.integers(41, len(e)))] = int(rng.integers(0, 256))
        streams.append(bytes(e))
        want.append(orc.decode_status(bytes(e), max_len=1 << 16))
    lens = np.array([len(s) for s in streams], np.uint64)
    offs = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.uint64)
    arena = np.frombuffer(b"".join(streams), np.uint8)
    caps = np.full(len(streams), 1 << 16, np.uint64)
    doffs = np.arange(len(streams), dtype=np.uint64) << np.uint64(16)
    d_dec, olens, st = codec.decode_batch(_dev(arena), np.stack([offs, lens], 1), np.stack([doffs, caps], 1),
                                          max_len=1 << 16, raise_on_error=False)
    dec = d_dec.cpu().numpy()
    for i, (ws, wb) in enumerate(want):
        assert st[i] == ws, (i, st[i], ws)
        if ws == 0:
            assert dec[int(doffs[i]):int(doffs[i]) + int(olens[i])].tobytes() == wb, i


def test_host_batches_in_chunks_match_single_pass(codec, orc):
    """Host-buffer batches of 32 MiB and more run as concurrent chunks; the
    streams, their placement and per-block statuses equal the one-pass
    device batch and the oracle, including a malformed stream late in the
    batch."""
    import torch

    data, spans = W.config1(nblocks=40, block=1 << 20, seed=4)
    h_src = torch.from_numpy(data.copy()).pin_memory().numpy()
    bound = codec.encode_bound(spans, 2)
    h_enc = torch.zeros(bound, dtype=torch.uint8).pin_memory().numpy()
    out, orders = codec.encode_batch_host(h_src, spans, 2, h_enc)
    d_out, sp, _ = codec.encode_batch(_dev(data), spans, 2)
    assert np.array_equal(out, sp)
    total = int(sp[-1, 0] + sp[-1, 1])
    assert np.array_equal(h_enc[:total], d_out[:total].cpu().numpy())
    for i in (0, 17, 39):
        o, l = int(sp[i, 0]), int(sp[i, 1])
        blk = data[int(spans[i, 0]):int(spans[i, 0] + spans[i, 1])].tobytes()
        e0, e1 = orc.encode(blk, 0), orc.encode(blk, 1)
        assert h_enc[o:o + l].tobytes() == (e1 if len(e1) < len(e0) else e0)
    # decode in chunks, with block 37 truncated
    enc = h_enc[:total].copy()
    bad = sp.copy()
    bad[37, 1] = bad[37, 1] // 2
    h_in = torch.from_numpy(enc).pin_memory().numpy()
    h_dec = torch.zeros(len(data), dtype=torch.uint8).pin_memory().numpy()
    old = codec.get_param("host_dec_chunks")
    codec.set_param("host_dec_chunks", 4)
    try:
        lens, st = codec.decode_batch_host(h_in, bad, spans, h_dec, raise_on_error=False)
    finally:
        codec.set_param("host_dec_chunks", old)
    stream37 = enc[int(bad[37, 0]):int(bad[37, 0] + bad[37, 1])].tobytes()
    assert st[37] == orc.decode_status(stream37)[0] != 0
    for i in range(40):
        if i == 37:
            continue
        assert st[i] == 0 and lens[i] == spans[i, 1]
        o, l = int(spans[i, 0]), int(spans[i, 1])
        assert np.array_equal(h_dec[o:o + l], data[o:o + l]), i


def test_launch_shapes_change_no_byte(codec):
    """Launch-shape parameters (fqxv_rans_ctx_set_param) move work between
    decoders and change grids; the streams and the decoded bytes stay the
    same."""
    import torch

    data, spans, _ = W.config2(nblocks=40, lo=1000, hi=400_000, seed=77)
    d_src = _dev(data)
    ref_out, ref_spans, _ = codec.encode_batch(d_src, spans, 2)
    ref = ref_out[:int(ref_spans[-1, 0] + ref_spans[-1, 1])].cpu().numpy()
    settings = [
        {"o1_four_max_streams": 0, "cta_cap_o1_wide": 1, "enc_run_ctas_per_sm": 4},
        {"o1_four_max_streams": 1 << 30, "cta_cap_o1_four": 1, "dense_edge_small": 0, "dense_edge_large": 0},
        {"cta_cap_o0": 1, "cta_cap_o1_small": 2, "cta_cap_o1_wide": 3, "dense_edge_small": 160 << 10,
         "dense_edge_large": 160 << 10},
        {"o1_top_exclusive": 0, "o1_top_max": 0, "enc_o1_keys": 0},
        {"o1_top_exclusive": 1, "o1_top_max": 5, "o1_top_latency_pct": 0},
        {"o1_top_exclusive": 1, "o1_top_max": 9, "o1_top_latency_pct": 0, "o1_top_small_per_sm": 2},
        {"o1_top_exclusive": 1, "o1_top_max": 1 << 20, "o1_top_latency_pct": 0, "enc_o1_keys": 0},
    ]
    defaults = {k: codec.get_param(k) for s in settings for k in s}
    try:
        for st in settings:
            for k, v in st.items():
                codec.set_param(k, v)
            out, osp, _ = codec.encode_batch(d_src, spans, 2)
            assert np.array_equal(osp, ref_spans)
            assert np.array_equal(out[:len(ref)].cpu().numpy(), ref)
            d_dec, lens, stt = codec.decode_batch(out, osp, spans)
            assert (stt == 0).all()
            assert torch.equal(d_dec[:len(data)], d_src[:len(data)])
    finally:
        for k, v in defaults.items():
            codec.set_param(k, v)
    with pytest.raises(Exception):
        codec.set_param("no_such_parameter", 1)
    with pytest.raises(Exception):
        codec.set_param("cta_cap_o0", 0)
