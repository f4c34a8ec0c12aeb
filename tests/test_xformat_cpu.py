"""The extended stream format's CPU definition (oracle/rans_x.c). PARITY
UNPINNED: the reference has no such format (it writes 32-way streams behind
a flag-less header, crates/fqxv-rans/src/scalar.rs:8-20), so these tests check
the definition against itself: every flag combination round trips, raw (CAT)
data passes through unchanged from the first version on, the selection keeps
the smallest candidate, reference streams are untouched, and malformed
streams give statuses, never a crash."""

import numpy as np
import pytest

from fqxv_b200 import workloads as W


def _inputs():
    rng = np.random.default_rng(0)
    return {
        "binned": W.binned_quality(20_000, 1).tobytes(),
        "full": W.full_quality(15_000, 2).tobytes(),
        "acgt": W.acgt(12_000, 3).tobytes(),
        "names": W.name_tokens(12_000, 4).tobytes(),
        "runs": np.repeat(rng.integers(0, 3, 800), rng.integers(1, 60, 800)).astype(np.uint8).tobytes(),
        "long_run": b"\x07" * 70_000 + b"\x01\x02" * 3,
        "bytes": bytes(range(256)) * 9,
        "random": rng.integers(0, 256, 9_000).astype(np.uint8).tobytes(),
        "one": b"Q",
        "three": b"ABC",
        "empty": b"",
    }


@pytest.mark.parametrize("name", list(_inputs()))
def test_every_flag_combination_round_trips(orc, name):
    data = _inputs()[name]
    nsym = len(set(data))
    for flags in range(64):
        # STRIPE codes its planes by the nested selection; other flags of
        # that level are ignored, PACK included
        if flags & orc.X_PACK and nsym > 16 and not flags & orc.X_STRIPE:
            with pytest.raises(orc.OracleError):
                orc.x_encode(data, flags)
            continue
        stream = orc.x_encode(data, flags)
        assert stream[0] == 0x80 | flags
        assert int.from_bytes(stream[1:9], "little") == len(data)
        assert orc.x_decode(stream, len(data)) == data, flags


def test_cat_passes_raw_bytes_through(orc):
    # the raw path: header, then the input bytes unchanged
    for data in (bytes(range(256)), b"", b"\x00" * 5, np.random.default_rng(1).bytes(4097)):
        stream = orc.x_encode(data, orc.X_CAT)
        assert stream == bytes([0x80 | orc.X_CAT]) + len(data).to_bytes(8, "little") + data
        assert orc.x_decode(stream, len(data)) == data


def test_four_way_cores_round_trip_and_differ_from_32_way(orc):
    data = W.binned_quality(50_000, 5).tobytes()
    for order in (0, 1):
        s4 = orc.x_encode(data, orc.X_N4 | order)
        s32 = orc.x_encode(data, order)
        assert s4 != s32
        # the 32-way core is the reference stream itself
        assert s32[17:] == orc.encode(data, order)
        assert orc.x_decode(s4, len(data)) == data


def test_selection_keeps_the_smallest_candidate(orc):
    for name, data in _inputs().items():
        stream, cand = orc.x_encode_best(data)
        assert orc.x_decode(stream, len(data)) == data
        sizes = [len(orc.encode(data, 0)), len(orc.encode(data, 1))]
        for flags in (orc.X_PACK, orc.X_PACK | 1, orc.X_RLE, orc.X_RLE | 1, orc.X_PACK | orc.X_RLE,
                      orc.X_PACK | orc.X_RLE | 1):
            sizes.append(len(orc.x_encode(data, flags)) if not (flags & orc.X_PACK and len(set(data)) > 16)
                         else 1 << 62)
        sizes.append(len(orc.x_encode(data, orc.X_STRIPE)) if len(data) >= 4 else 1 << 62)
        sizes.append(len(orc.x_encode(data, orc.X_CAT)))
        assert len(stream) == min(sizes), name
        assert cand == sizes.index(min(sizes)), name


def test_reference_streams_decode_unchanged(orc, golden):
    for _, stream in golden:
        assert orc.x_decode(stream) == orc.decode(stream)


def test_malformed_streams_give_statuses(orc):
    rng = np.random.default_rng(9)
    seen = set()
    for data in (_inputs()["binned"][:3000], _inputs()["runs"][:3000], _inputs()["full"][:2000]):
        for flags in (0, 1, 2, 3, 4, 8, 9, 10, 16, 24, 25, 32, 40):
            if flags & 16 and len(set(data)) > 16:
                continue
            base = bytearray(orc.x_encode(data, flags))
            for _ in range(60):
                m = bytearray(base)
                if rng.random() < 0.4:
                    m = m[:int(rng.integers(1, len(m)))]
                else:
                    for _ in range(int(rng.integers(1, 4))):
                        m[int(rng.integers(0, len(m)))] = int(rng.integers(0, 256))
                st = orc.x_decode_status(bytes(m), len(data) + 64)
                assert st in (0, 1, 2, 3, 4, 5, 6, 9)
                seen.add(st)
    assert {1, 9} <= seen
