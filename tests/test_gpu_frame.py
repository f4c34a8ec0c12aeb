"""GPU parity of the CRC-32C / block-frame row against the oracle
(oracle/frame_oracle.c, the restatement of crates/fqxv/src/crc.rs and
crates/fqxv/src/container/block.rs) and against the CRCs the reference stored
in its golden archives. Integer work: every CRC, frame byte, status and
offset must be identical."""

import json
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def codec():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from fqxv_b200.batch import Codec

    c = Codec(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def crc_golden():
    with open(os.path.join(GOLDEN, "fixture_crcs.json")) as f:
        recs = json.load(f)["records"]
    with open(os.path.join(GOLDEN, "fixture_crcs.bin"), "rb") as f:
        blob = f.read()
    return recs, blob


def _dev(a):
    import torch

    return torch.from_numpy(np.array(a, dtype=np.uint8, copy=True)).to("cuda")


def _random_spans(rng, size, n, max_len):
    spans = []
    for _ in range(n):
        ln = int(min(size, rng.integers(0, max_len + 1)))
        off = int(rng.integers(0, size - ln + 1))
        spans.append((off, ln))
    return np.array(spans, dtype=np.uint64).reshape(-1, 2)


def test_known_answers(codec):
    from fqxv_b200 import frame

    assert frame.crc32c(b"") == 0
    assert frame.crc32c(b"123456789") == 0xE3069283


def test_crc_batch_matches_oracle(codec, orc):
    rng = np.random.default_rng(11)
    size = 6 << 20
    data = rng.integers(0, 256, size, dtype=np.uint8)
    d = _dev(data)
    lens = [0, 1, 2, 3, 4, 5, 7, 8, 9, 31, 127, 128, 129, 255, 256, 257, 4095, 4096, 4097, 65535,
            65536, 65537, 200000, (1 << 20) + 3, 5 << 20]
    spans = [(int(rng.integers(0, size - ln + 1)), ln) for ln in lens]
    spans += [(k, 1000) for k in range(8)]                      # every start alignment
    spans += list(map(tuple, _random_spans(rng, size, 400, 70000)))
    spans = np.array(spans, dtype=np.uint64)
    got = codec.crc32c_batch(d, spans)
    want = [orc.crc32c(data[int(o):int(o) + int(ln)]) for o, ln in spans]
    assert list(got) == want
    # a device pointer that is not 4-byte aligned
    got1 = codec.crc32c_batch(d[1:], spans[spans[:, 0] + spans[:, 1] < size - 1])
    sub = spans[spans[:, 0] + spans[:, 1] < size - 1]
    assert list(got1) == [orc.crc32c(data[1 + int(o):1 + int(o) + int(ln)]) for o, ln in sub]
    # host form
    got2 = codec.crc32c_batch_host(data, spans)
    assert list(got2) == want


def test_crc_matches_every_stored_golden_crc(codec, crc_golden):
    recs, blob = crc_golden
    kept = [r for r in recs if r["bin_offset"] is not None]
    arr = np.frombuffer(blob, dtype=np.uint8)
    spans = np.array([(r["bin_offset"], r["length"]) for r in kept], dtype=np.uint64)
    got = codec.crc32c_batch(_dev(arr), spans)
    assert list(got) == [r["crc"] for r in kept]
    assert {r["kind"] for r in kept} >= {"header", "block_frame", "stream_loc", "whole_file", "footer",
                                          "framed_slice"}


def test_large_span_and_combine(codec, orc):
    """Full-size property: a 512 MiB span against the oracle, and the CRC of
    the whole equals crc32c_combine of the CRCs of its parts."""
    from fqxv_b200 import frame

    rng = np.random.default_rng(5)
    n = 512 << 20
    data = rng.integers(0, 256, n, dtype=np.uint8)
    d = _dev(data)
    cuts = [0, 3, 1 << 20, (200 << 20) + 1, n]
    spans = np.array([(0, n)] + [(a, b - a) for a, b in zip(cuts, cuts[1:])], dtype=np.uint64)
    got = codec.crc32c_batch(d, spans)
    assert int(got[0]) == orc.crc32c(data)
    c = int(got[1])
    for (a, b), part in zip(zip(cuts[1:], cuts[2:]), got[2:]):
        c = frame.crc32c_combine(c, int(part), b - a)
    assert c == int(got[0])


def test_frame_blocks_match_oracle(codec, orc):
    import torch

    rng = np.random.default_rng(3)
    size = 3 << 20
    data = rng.integers(0, 256, size, dtype=np.uint8)
    spans = _random_spans(rng, size, 300, 40000)
    spans[5] = (17, 0)                              # empty payload
    spans[6] = (1, 3)
    spans = np.concatenate([spans, np.array([[0, 2 << 20], [5, (1 << 20) + 7]], dtype=np.uint64)])
    for terminate in (False, True):
        want, wfo, wcrc = orc.frame_blocks(data, spans[:, 0], spans[:, 1], terminate)
        d_dst, fo, crcs, total = codec.frame_blocks(_dev(data), spans, terminate)
        torch.cuda.synchronize()
        assert total == len(want)
        assert d_dst[:total].cpu().numpy().tobytes() == want
        assert list(fo) == list(wfo) and list(crcs) == list(wcrc)
    # misaligned destination and source pointers
    d_src = _dev(data)
    buf = torch.zeros(len(want) + 8, dtype=torch.uint8, device="cuda")
    sub = spans[spans[:, 0] + spans[:, 1] < size - 3]
    want2, _, _ = orc.frame_blocks(data[3:], sub[:, 0], sub[:, 1], True)
    _, _, _, total = codec.frame_blocks(d_src[3:], sub, True, d_dst=buf[5:])
    torch.cuda.synchronize()
    out = buf.cpu().numpy()
    assert out[5:5 + total].tobytes() == want2
    assert not out[:5].any() and not out[5 + total:].any()   # nothing written outside
    # host form
    h_dst = np.zeros(len(want), dtype=np.uint8)
    fo, crcs, total = codec.frame_blocks_host(data, spans, h_dst, True)
    assert h_dst[:total].tobytes() == want


def test_read_blocks_match_oracle(codec, orc):
    rng = np.random.default_rng(9)
    payloads = [rng.integers(0, 256, int(n), dtype=np.uint8).tobytes()
                for n in rng.integers(1, 30000, 120)]
    src = np.frombuffer(b"".join(payloads), dtype=np.uint8)
    lens = [len(p) for p in payloads]
    offs = np.concatenate([[0], np.cumsum(lens)[:-1]])
    fr, _, _ = orc.frame_blocks(src, offs, lens, True)
    fr = np.frombuffer(fr + b"trailing footer bytes", dtype=np.uint8)

    def check(buf, max_frames=None):
        first, pay, crcs, st, consumed, term = orc.read_blocks(buf, max_frames)
        for got in (codec.read_blocks(_dev(buf), max_frames=max_frames),
                    codec.read_blocks_host(np.ascontiguousarray(buf), max_frames=max_frames)):
            gpay, gcrcs, gst, gcons, gterm = got
            assert np.array_equal(gpay, pay) and list(gst) == list(st)
            assert gcons == consumed and gterm == term
            assert list(gcrcs) == list(crcs)
        return first, st

    first, st = check(fr)
    assert first == 0 and len(st) == 120
    check(fr, max_frames=7)
    # payload corruption in three frames: CORRUPT, walk continues
    bad = fr.copy()
    for k in (0, 50, 119):
        bad[int(offs[k]) + 16 * (k + 1) + int(lens[k]) // 2] ^= 0x40
    first, st = check(bad)
    assert first == 33 and list(np.nonzero(st)[0]) == [0, 50, 119]
    # bad marker, truncations, oversize length
    bad = fr.copy()
    bad[int(offs[60]) + 16 * 60 + 2] = 0
    first, st = check(bad)
    assert first == 34 and len(st) == 61
    for cut in (3, 4, 11, 12, 15, 16, 100, int(offs[30]) + 16 * 30 + 20, len(fr) - 21 - 12 - 5):
        check(fr[:cut])
    big = np.frombuffer(b"FQXB" + ((1 << 31) + 9).to_bytes(8, "little") + bytes(40), dtype=np.uint8)
    assert check(big)[0] == 35


def test_read_blocks_chain_paths(codec, orc):
    """Walks past the serial head: the marker scan and chain (fake markers
    planted inside payloads, some with lengths that land on real frame
    starts), max_frames cuts inside the chain, and more marker hits than the
    chain holds (the serial fallback)."""
    rng = np.random.default_rng(21)

    def frames(payloads, terminate=True):
        src = np.frombuffer(b"".join(payloads), dtype=np.uint8)
        lens = [len(p) for p in payloads]
        offs = np.concatenate([[0], np.cumsum(lens)[:-1]])
        return orc.frame_blocks(src, offs, lens, terminate)[0]

    def check(buf, max_frames=None):
        buf = np.frombuffer(buf, dtype=np.uint8) if isinstance(buf, bytes) else buf
        first, pay, crcs, st, consumed, term = orc.read_blocks(buf, max_frames)
        gpay, gcrcs, gst, gcons, gterm = codec.read_blocks(_dev(buf), max_frames=max_frames)
        assert np.array_equal(gpay, pay) and list(gst) == list(st)
        assert gcons == consumed and gterm == term and list(gcrcs) == list(crcs)
        return st

    pls = []
    for k in range(2000):
        b = bytearray(rng.integers(0, 256, int(rng.integers(20, 3000)), dtype=np.uint8).tobytes())
        if k % 5 == 0:
            q = int(rng.integers(0, len(b) - 16))
            b[q:q + 4] = b"FQXB"
            b[q + 4:q + 12] = int(rng.choice([0, 5, len(b) - q - 16, (1 << 31) + 3])).to_bytes(8, "little")
        pls.append(bytes(b))
    fr = frames(pls)
    assert len(check(fr)) == 2000
    for mf in (33, 40, 1000, 1999, 2000, 2001):
        check(fr, max_frames=mf)
    bad = bytearray(fr)
    pos = sum(16 + len(p) for p in pls[:1500])
    bad[pos] = ord("G")
    assert list(np.nonzero(check(bytes(bad)))[0]) == [1500]
    check(fr[:pos + 10])
    check(fr[:-12] + b"tail")        # no terminator, clean end then junk
    many = frames([bytes([k & 255]) * 3 for k in range(9000)])
    assert len(check(many)) == 9000


def test_read_blocks_golden_archive(codec, crc_golden):
    recs, blob = crc_golden
    arr = np.frombuffer(blob, dtype=np.uint8)
    for fx in ("plain_se", "paired_labels"):
        hdr = next(r for r in recs if r["fixture"] == fx and r["kind"] == "header")
        frames = [r for r in recs if r["fixture"] == fx and r["kind"] == "block_frame"]
        footer = next(r for r in recs if r["fixture"] == fx and r["kind"] == "footer")
        start = hdr["bin_offset"] + hdr["length"] + 4
        region = arr[start:footer["bin_offset"]]
        pay, crcs, st, consumed, term = codec.read_blocks(_dev(region))
        assert term and consumed == len(region) and not st.any()
        assert list(crcs) == [f["crc"] for f in frames]


def test_payload_stream_locs(codec, orc, crc_golden):
    recs, blob = crc_golden
    arr = np.frombuffer(blob, dtype=np.uint8)
    frames = [r for r in recs if r["kind"] == "block_frame" and r["bin_offset"] is not None]
    spans = np.array([(r["bin_offset"], r["length"]) for r in frames], dtype=np.uint64)
    d = _dev(arr)
    locs, st = codec.payload_stream_locs(d, spans)
    assert not st.any()
    for i, fr in enumerate(frames):
        want = [r for r in recs if r["fixture"] == fr["fixture"] and r["kind"] == "stream_loc"]
        base = fr["offset"] - fr["bin_offset"]          # archive offset of arr[0] for this fixture
        got = [(int(l["offset"]) + base, int(l["len"]), int(l["crc"])) for l in locs[i]]
        assert got == [(w["offset"], w["length"], w["crc"]) for w in want]
    # random payloads, some truncated
    rng = np.random.default_rng(2)
    pls = []
    for k in range(50):
        streams = [rng.integers(0, 256, int(rng.integers(0, 5000)), dtype=np.uint8).tobytes() for _ in range(3)]
        p = bytes(24) + (k).to_bytes(4, "little") + b"".join(len(s).to_bytes(4, "little") + s for s in streams)
        if k % 7 == 3:
            p = p[:int(rng.integers(0, len(p)))]
        pls.append(p)
    src = np.frombuffer(b"".join(pls), dtype=np.uint8)
    lens = [len(p) for p in pls]
    offs = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.uint64)
    sp = np.stack([offs, np.array(lens, dtype=np.uint64)], axis=1)
    locs, st = codec.payload_stream_locs(_dev(src), sp, base=1000)
    for i, p in enumerate(pls):
        rc, want = orc.payload_stream_locs(p, 0)
        assert st[i] == rc
        if rc == 0:
            got = [(int(l["offset"]) - 1000 - int(offs[i]), int(l["len"]), int(l["crc"])) for l in locs[i]]
            assert got == [(o - 16, ln, c) for o, ln, c in want]


def test_reference_shaped_module(codec):
    from fqxv_b200 import frame

    payloads = [b"alpha" * 100, b"", b"b", bytes(range(256)) * 9]
    buf = frame.write_blocks([p for p in payloads if p], terminate=True)
    assert frame.read_blocks(buf) == [p for p in payloads if p]
    payload, pos = frame.read_block(buf)
    assert payload == payloads[0] and pos == 16 + 500
    bad = bytearray(buf)
    bad[16 + 500 + 16] ^= 1
    with pytest.raises(frame.Corrupt) as e:
        frame.read_blocks(bytes(bad))
    assert str(e.value) == "corrupted fqxv data: block 1 (crc mismatch)"
    bad = bytearray(buf)
    bad[16 + 500] = ord("X")
    with pytest.raises(frame.Corrupt) as e:
        frame.read_blocks(bytes(bad))
    assert e.value.what == "block 1 (bad sync marker)"
    with pytest.raises(frame.Truncated):
        frame.read_blocks(buf[:30])
