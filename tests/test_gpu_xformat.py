"""The extended stream format on the GPU against its CPU definition
(oracle/rans_x.c), byte for byte. PARITY UNPINNED against the reference,
which has no such format; the reference's own streams keep decoding."""

import numpy as np
import pytest

from fqxv_b200 import rans
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


def _arena(blobs):
    lens = np.array([len(b) for b in blobs], dtype=np.uint64)
    offs = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.uint64) if len(blobs) else np.zeros(0, np.uint64)
    arena = np.frombuffer(b"".join(blobs) or b"\0", dtype=np.uint8).copy()
    return arena, np.stack([offs, lens], 1)


def _dev(a):
    import torch

    return torch.from_numpy(np.array(a, dtype=np.uint8, copy=True)).to("cuda")


def _blobs(seed=0, small=False):
    rng = np.random.default_rng(seed)
    k = 1 if small else 3
    return [
        W.binned_quality(20_000 * k, seed + 1).tobytes(),
        W.full_quality(9_000 * k, seed + 2).tobytes(),
        W.acgt(11_000 * k, seed + 3).tobytes(),
        W.name_tokens(7_000 * k, seed + 4).tobytes(),
        np.repeat(rng.integers(0, 3, 500), rng.integers(1, 50, 500)).astype(np.uint8).tobytes(),
        b"\x05" * 40_000,
        bytes(range(256)) * 3,
        b"AB",
        b"",
    ]


def _check_encode(codec, orc, blobs, flags):
    arena, spans = _arena(blobs)
    d_out, out_spans, choice = codec.x_encode_batch(_dev(arena), spans, flags)
    out = d_out.cpu().numpy()
    streams = []
    for i, b in enumerate(blobs):
        o, ln = int(out_spans[i, 0]), int(out_spans[i, 1])
        got = out[o:o + ln].tobytes()
        if flags == 0x40:
            want, cand = orc.x_encode_best(b)
            assert int(choice[i]) == cand, i
        else:
            want = orc.x_encode(b, flags)
        assert got == want, (i, flags, len(b))
        streams.append(got)
    return streams


@pytest.mark.parametrize("flags", [0, 1, 2, 3, 8, 9, 10, 11, 32, 33, 40])
def test_flags_match_the_definition(codec, orc, flags):
    blobs = _blobs(flags)
    streams = _check_encode(codec, orc, blobs, flags)
    arena, spans = _arena(streams)
    _, rsp = _arena(blobs)
    d_dec, lens, st = codec.x_decode_batch(_dev(arena), spans, rsp)
    assert (st == 0).all() and (lens == rsp[:, 1]).all()
    assert d_dec[:int(rsp[:, 1].sum())].cpu().numpy().tobytes() == b"".join(blobs)


@pytest.mark.parametrize("flags", [16, 17, 18, 24, 25, 26, 27, 48])
def test_pack_flags_match_the_definition(codec, orc, flags):
    blobs = [b for b in _blobs(flags) if len(set(b)) <= 16]
    streams = _check_encode(codec, orc, blobs, flags)
    arena, spans = _arena(streams)
    _, rsp = _arena(blobs)
    d_dec, lens, st = codec.x_decode_batch(_dev(arena), spans, rsp)
    assert (st == 0).all()
    assert d_dec[:int(rsp[:, 1].sum())].cpu().numpy().tobytes() == b"".join(blobs)


def test_stripe_matches_the_definition(codec, orc):
    blobs = _blobs(4, small=True) + [b"x", b"xyz"]
    streams = _check_encode(codec, orc, blobs, 4)
    arena, spans = _arena(streams)
    _, rsp = _arena(blobs)
    d_dec, lens, st = codec.x_decode_batch(_dev(arena), spans, rsp)
    assert (st == 0).all()
    assert d_dec[:int(rsp[:, 1].sum())].cpu().numpy().tobytes() == b"".join(blobs)


def test_selection_matches_the_definition(codec, orc):
    blobs = _blobs(7, small=True)
    streams = _check_encode(codec, orc, blobs, 0x40)
    arena, spans = _arena(streams)
    _, rsp = _arena(blobs)
    d_dec, lens, st = codec.x_decode_batch(_dev(arena), spans, rsp)
    assert (st == 0).all()
    assert d_dec[:int(rsp[:, 1].sum())].cpu().numpy().tobytes() == b"".join(blobs)


def test_config0_four_way_full_size(codec, orc):
    # config 0 as named: one 1 MiB block of binned quality, order-0, 4-way
    data, spans = W.config0()
    blob = data.tobytes()
    streams = _check_encode(codec, orc, [blob], 0x02)
    d_dec, lens, st = codec.x_decode_batch(_dev(np.frombuffer(streams[0], np.uint8)), [[0, len(streams[0])]],
                                           [[0, len(blob)]])
    assert (st == 0).all() and d_dec[:len(blob)].cpu().numpy().tobytes() == blob


def test_oracle_streams_decode_on_gpu(codec, orc):
    blobs = _blobs(11, small=True)
    streams = []
    for i, b in enumerate(blobs):
        flags = [0, 1, 2, 3, 8, 11, 32, 40, 0x40][i % 9]
        streams.append(orc.x_encode_best(b)[0] if flags == 0x40 else orc.x_encode(b, flags))
    streams += [orc.encode(b, 1) for b in blobs[:3]]   # the reference format, unchanged
    blobs = blobs + blobs[:3]
    arena, spans = _arena(streams)
    _, rsp = _arena(blobs)
    d_dec, lens, st = codec.x_decode_batch(_dev(arena), spans, rsp)
    assert (st == 0).all()
    assert d_dec[:int(rsp[:, 1].sum())].cpu().numpy().tobytes() == b"".join(blobs)


def test_cat_passthrough_on_gpu(codec, orc):
    blobs = [bytes(range(256)), np.random.default_rng(3).bytes(5000), b"\x00" * 17, b""]
    streams = _check_encode(codec, orc, blobs, 32)
    for b, s in zip(blobs, streams):
        assert s[9:] == b


def test_truncated_streams_match_the_definition(codec, orc):
    rng = np.random.default_rng(2)
    base = [W.binned_quality(3000, 5).tobytes(), np.repeat(rng.integers(0, 3, 80), rng.integers(1, 30, 80)).astype(
        np.uint8).tobytes()]
    streams, caps = [], []
    for b in base:
        for flags in (0, 2, 3, 8, 24, 32, 4):
            s = orc.x_encode(b, flags)
            for cut in sorted(set(int(c) for c in rng.integers(1, len(s), 6))):
                streams.append(s[:cut])
                caps.append(len(b))
    arena, spans = _arena(streams)
    offs = np.concatenate([[0], np.cumsum(caps)[:-1]]).astype(np.uint64)
    rsp = np.stack([offs, np.array(caps, np.uint64)], 1)
    _, lens, st = codec.x_decode_batch(_dev(arena), spans, rsp, raise_on_error=False)
    want = [orc.x_decode_status(s, c) for s, c in zip(streams, caps)]
    assert list(st) == want


@pytest.mark.parametrize("flags", [0x02, 0x03])
def test_four_way_cores_ragged_lengths(codec, orc, flags):
    """4-way cores whose length is not a multiple of four, and long enough
    that the decoder's four-lane rounds run before the serial remainder:
    the GPU streams equal the definition's and decode back."""
    blobs = [W.binned_quality(n, 700 + n % 7).tobytes() for n in (4, 5, 6, 7, 8001, 8002, 8003, 65537, 100_003)]
    blobs += [W.full_quality(n, 710 + n % 5).tobytes() for n in (9, 70_001, 131_075)]
    streams = _check_encode(codec, orc, blobs, flags)
    arena, spans = _arena(streams)
    _, ospans = _arena(blobs)
    d_dec, lens, st = codec.x_decode_batch(_dev(arena), spans, ospans)
    dec = d_dec.cpu().numpy()
    for i, b in enumerate(blobs):
        assert st[i] == 0 and int(lens[i]) == len(b)
        o = int(ospans[i, 0])
        assert dec[o:o + len(b)].tobytes() == b, i
