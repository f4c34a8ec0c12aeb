"""CPU checks of the CRC-32C / block-frame row: the oracle against the
reference's known answers (crates/fqxv/src/crc.rs:196-262) and against every
CRC the reference stored in its golden archives; the oracle's frame walk
against the read_block rules (crates/fqxv/src/container/block.rs:1209-1254);
and the library's host-only arithmetic (fqxv_crc32c_combine) against the
oracle."""

import json
import os
import random

import numpy as np
import pytest

from conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def crc_golden():
    with open(os.path.join(GOLDEN, "fixture_crcs.json")) as f:
        recs = json.load(f)["records"]
    with open(os.path.join(GOLDEN, "fixture_crcs.bin"), "rb") as f:
        blob = f.read()
    return recs, blob


def rec_bytes(blob, r):
    return blob[r["bin_offset"]:r["bin_offset"] + r["length"]]


# ---- crc.rs tests, restated ---------------------------------------------------

def test_known_answers(orc):
    # crc.rs:201-205
    assert orc.crc32c(b"") == 0
    assert orc.crc32c(b"123456789") == 0xE3069283


def test_incremental_matches_oneshot(orc):
    # crc.rs:208-214: Hasher::update in pieces == crc32c of the whole
    data = b"the quick brown fox jumps over the lazy dog"
    L = orc.lib()
    a, pa = orc._buf(data[:10])
    b, pb = orc._buf(data[10:])
    st = L.orc_crc32c_update(0xFFFFFFFF, pa, a.size)
    st = L.orc_crc32c_update(st, pb, b.size)
    assert st ^ 0xFFFFFFFF == orc.crc32c(data)


def test_detects_single_bit_flip(orc):
    assert orc.crc32c(b"ACGTACGTACGT") != orc.crc32c(b"ACGTACGTACGA")


def test_combine_reassembles_split_buffer(orc):
    # crc.rs:228-236 and :239-242
    data = b"the quick brown fox jumps over the lazy dog"
    for k in range(len(data) + 1):
        a, b = data[:k], data[k:]
        assert orc.crc32c_combine(orc.crc32c(a), orc.crc32c(b), len(b)) == orc.crc32c(data)
    a = orc.crc32c(b"123456789")
    assert orc.crc32c_combine(a, orc.crc32c(b""), 0) == a


def test_combine_matches_concatenation_random(orc):
    # crc.rs:244-255 (proptest), with seeded inputs
    rng = random.Random(7)
    for _ in range(200):
        a = bytes(rng.randrange(256) for _ in range(rng.randrange(0, 300)))
        b = bytes(rng.randrange(256) for _ in range(rng.randrange(0, 300)))
        assert orc.crc32c_combine(orc.crc32c(a), orc.crc32c(b), len(b)) == orc.crc32c(a + b)


# ---- the pin: CRCs stored in the reference's golden archives -----------------

def test_oracle_matches_every_stored_crc(orc, crc_golden):
    recs, blob = crc_golden
    kinds = set()
    checked = 0
    for r in recs:
        if r["bin_offset"] is None:
            continue
        assert orc.crc32c(rec_bytes(blob, r)) == r["crc"], r
        kinds.add(r["kind"])
        checked += 1
    assert checked >= 25
    assert kinds >= {"header", "block_frame", "stream_loc", "whole_file", "footer", "framed_slice"}


def test_whole_file_crc_by_combining_frames(orc, crc_golden):
    # format.rs:318-338: whole_file_crc is the running CRC of every byte
    # before it; rebuilt here from the CRCs of consecutive ranges.
    recs, blob = crc_golden
    for fx in ("plain_se", "paired_labels"):
        whole = next(r for r in recs if r["fixture"] == fx and r["kind"] == "whole_file")
        data = blob[whole["bin_offset"]:whole["bin_offset"] + whole["length"]]
        cuts = [0, 25, len(data) // 3, len(data) // 2, len(data)]
        crc = orc.crc32c(data[:0])
        for a, b in zip(cuts, cuts[1:]):
            crc = orc.crc32c_combine(crc, orc.crc32c(data[a:b]), b - a)
        assert crc == whole["crc"]


def test_oracle_walks_the_golden_block_region(orc, crc_golden):
    recs, blob = crc_golden
    for fx in ("plain_se", "paired_labels"):
        hdr = next(r for r in recs if r["fixture"] == fx and r["kind"] == "header")
        frames = [r for r in recs if r["fixture"] == fx and r["kind"] == "block_frame"]
        footer = next(r for r in recs if r["fixture"] == fx and r["kind"] == "footer")
        start = hdr["bin_offset"] + hdr["length"] + 4
        region = blob[start:footer["bin_offset"]]
        first, pay, crcs, st, consumed, term = orc.read_blocks(region)
        assert first == 0 and term and consumed == len(region)
        assert [int(c) for c in crcs] == [f["crc"] for f in frames]
        assert all(int(p[0]) + start == f["bin_offset"] for p, f in zip(pay, frames))


def test_oracle_stream_locs_match_the_footer(orc, crc_golden):
    recs, blob = crc_golden
    for fx in ("plain_se", "paired_labels"):
        frame = next(r for r in recs if r["fixture"] == fx and r["kind"] == "block_frame")
        locs = [r for r in recs if r["fixture"] == fx and r["kind"] == "stream_loc"]
        payload = rec_bytes(blob, frame)
        frame_start = frame["offset"] - 16
        rc, got = orc.payload_stream_locs(payload, frame_start)
        assert rc == 0
        assert got == [(l["offset"], l["length"], l["crc"]) for l in locs]


# ---- the oracle's frame rules (block.rs:110-142, :1209-1254) ---------------------

def _frames(orc, payloads, terminate=True):
    src = np.frombuffer(b"".join(payloads) or b"\0", dtype=np.uint8)
    lens = [len(p) for p in payloads]
    offs = np.concatenate([[0], np.cumsum(lens)[:-1]]) if payloads else []
    return orc.frame_blocks(src, offs, lens, terminate)


def test_frame_layout(orc):
    fr, fo, crcs = _frames(orc, [b"abc", b"defgh"])
    assert fr[:4] == b"FQXB" and int.from_bytes(fr[4:12], "little") == 3
    assert int.from_bytes(fr[12:16], "little") == orc.crc32c(b"abc") == crcs[0]
    assert fr[16:19] == b"abc" and list(fo) == [0, 19]
    assert fr[-12:] == b"FQXB" + bytes(8)


def test_walk_rules(orc):
    fr, _, _ = _frames(orc, [b"x" * 40, b"y" * 7, b"z" * 100], terminate=True)
    first, pay, crcs, st, consumed, term = orc.read_blocks(fr)
    assert first == 0 and term and consumed == len(fr) and len(st) == 3
    # clean end without a terminator; fewer than 4 bytes left is a clean end
    fr2, _, _ = _frames(orc, [b"a" * 5], terminate=False)
    assert orc.read_blocks(fr2 + b"FQX")[0] == 0
    # bad marker
    bad = bytearray(fr)
    bad[56 + 1] = ord("X")  # second frame's marker
    first, pay, crcs, st, consumed, term = orc.read_blocks(bytes(bad))
    assert first == 34 and list(st) == [0, 34] and consumed == 56 and not term
    # payload corruption: CORRUPT, and the walk goes on
    bad = bytearray(fr)
    bad[20] ^= 1
    first, pay, crcs, st, consumed, term = orc.read_blocks(bytes(bad))
    assert first == 33 and list(st) == [33, 0, 0] and term
    # truncations at every cut point of the last frame
    for cut in range(len(fr) - 12 - 116 + 1, len(fr) - 12):
        first, pay, crcs, st, consumed, term = orc.read_blocks(fr[:cut])
        left = cut - (len(fr) - 12 - 116)
        if left < 4:
            assert first == 0 and len(st) == 2
        else:
            assert first == 32 and st[-1] == 32, cut
    # declared length above MAX_BLOCK_PAYLOAD
    big = b"FQXB" + ((1 << 31) + 1).to_bytes(8, "little") + bytes(4) + b"q" * 10
    assert orc.read_blocks(big)[0] == 35
    # max_frames
    first, pay, crcs, st, consumed, term = orc.read_blocks(fr, max_frames=2)
    assert len(st) == 2 and consumed == 56 + 16 + 7 and not term


def test_stream_locs_truncation(orc):
    body = bytes(24) + (7).to_bytes(4, "little")
    streams = [b"names", b"seq!", b"qq"]
    payload = body + b"".join(len(s).to_bytes(4, "little") + s for s in streams)
    rc, locs = orc.payload_stream_locs(payload, 1000)
    assert rc == 0
    assert [l[1] for l in locs] == [5, 4, 2]
    assert locs[0][0] == 1000 + 16 + 28 + 4
    assert [l[2] for l in locs] == [orc.crc32c(s) for s in streams]
    for cut in range(len(payload)):
        assert orc.payload_stream_locs(payload[:cut], 0)[0] == 32


# ---- library host arithmetic and symbols ---------------------------------------

def test_library_combine_matches_oracle(orc):
    from fqxv_b200 import frame

    rng = random.Random(3)
    for _ in range(300):
        a, b = rng.getrandbits(32), rng.getrandbits(32)
        n = rng.choice([0, 1, 3, 4, 127, 4096, rng.getrandbits(20), rng.getrandbits(40), (1 << 63) + 5])
        assert frame.crc32c_combine(a, b, n) == orc.crc32c_combine(a, b, n)


def test_frame_status_numbering_matches_oracle():
    import re

    text = open(os.path.join(ROOT, "include", "fqxv_frame_gpu.h")).read()
    o = open(os.path.join(ROOT, "oracle", "rans_oracle.h")).read()
    pairs = dict(re.findall(r"FQXV_FRAME_(E_\w+) = (\d+)", text))
    opairs = dict(re.findall(r"ORC_FRAME_(E_\w+) = (\d+)", o))
    assert pairs == opairs and len(pairs) == 4
