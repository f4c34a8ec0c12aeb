"""GPU parity: the CUDA path against the oracle, through the C ABI.

Bit-exact is the bar: every stream the GPU writes equals the oracle's
(= the reference encoder's) bytes, every stream decodes to the input, and
malformed input yields the reference's error kind. Mirrors the reference's
own tests (crates/fqxv-rans/src/lib.rs:261-604).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from fqxv_b200 import rans

    return rans


def _check(gpu, orc, data, orders=(0, 1)):
    data = bytes(data)
    for order in orders:
        ref = orc.encode(data, order)
        got = gpu.encode(data, gpu.Order(order))
        assert got == ref, (order, len(data))
        assert gpu.decode(ref) == data, (order, len(data))


def test_golden_streams(gpu, orc, golden):
    for meta, stream in golden:
        dec = gpu.decode(stream)
        assert dec == orc.decode(stream)
        assert gpu.encode(dec, gpu.Order(stream[0])) == stream, meta["stream"]


def test_roundtrip_empty_single_allsame(gpu, orc):
    _check(gpu, orc, b"")
    _check(gpu, orc, b"Q")
    _check(gpu, orc, b"A" * 1000)


def test_roundtrip_short_and_odd_lengths(gpu, orc):
    for n in [1, 2, 31, 32, 33, 63, 64, 65, 100, 511, 512, 513, 1000]:
        _check(gpu, orc, bytes((i * 7 + 3) & 0xFF for i in range(n)))


def test_full_alphabet_and_arbitrary_bytes(gpu, orc):
    _check(gpu, orc, bytes(i & 0xFF for i in range(10_000)))
    rng = np.random.default_rng(11)
    for n in [257, 4096, 70_001]:
        _check(gpu, orc, rng.integers(0, 256, n).astype(np.uint8).tobytes())


def test_skewed_frequency_regimes(gpu, orc):
    # lib.rs:439-447: a dominant symbol (freq > 2048, the exact-division
    # regime), a single symbol (freq == 4096) and a two-symbol skew.
    cases = [b"A" * 60_000 + bytes(ord("B") + (i % 20) for i in range(4000)), b"Q" * 40_000,
             bytes(ord("!") + 7 * (i % 3 == 0) for i in range(80_000))]
    for c in cases:
        _check(gpu, orc, c)


def test_random_small_alphabets(gpu, orc):
    rng = np.random.default_rng(5)
    for _ in range(25):
        n = int(rng.integers(0, 5000))
        k = int(rng.integers(1, 41))
        _check(gpu, orc, rng.integers(0, k, n).astype(np.uint8).tobytes())


def test_order1_beats_order0_and_best_modes(gpu, orc):
    x = 0
    data = bytearray()
    for i in range(100_000):
        x = (x + (i % 4)) & 0xFF
        data.append(ord("A") + (x % 4))
    data = bytes(data)
    e0, e1 = orc.encode(data, 0), orc.encode(data, 1)
    assert len(e1) < len(e0)
    assert gpu.encode(data, gpu.Order.BestTie0) == e1
    # ties: both orders give 9 bytes on empty input
    assert gpu.encode(b"", gpu.Order.BestTie0) == bytes(9)
    assert gpu.encode(b"", gpu.Order.BestTie1) == b"\x01" + bytes(8)
    small = b"AB"  # order-0 wins (order-1 carries two tables)
    assert gpu.encode(small, gpu.Order.BestTie1) == orc.encode(small, 0)


def test_decode_bounded(gpu, orc):
    enc = bytearray(orc.encode(b"A" * 64, 0))
    bomb = bytearray(enc)
    bomb[1:9] = (1 << 31).to_bytes(8, "little")
    with pytest.raises(gpu.Malformed) as e:
        gpu.decode_bounded(bytes(bomb), 1 << 20)
    assert e.value.status == 7
    assert gpu.decode_bounded(bytes(enc), 1 << 20) == b"A" * 64
    with pytest.raises(gpu.Malformed):
        gpu.decode_bounded(bytes(enc[:1]), 1 << 20)


def test_malformed_tables_and_huge_length(gpu, orc):
    src = b"\x00" + (1).to_bytes(8, "little")
    freq = np.zeros(256, np.uint16)
    freq[0] = 4096 + 100
    with pytest.raises(gpu.Malformed) as e:
        gpu.decode(src + freq.tobytes())
    assert e.value.status == 3
    src = b"\x00" + (2**64 - 1).to_bytes(8, "little")
    freq[0] = 4096
    with pytest.raises(gpu.Malformed) as e:
        gpu.decode(src + freq.tobytes() + bytes(128))
    assert e.value.status == 6


def _status(fn, *a):
    try:
        return 0, fn(*a)
    except Exception as ex:  # noqa: BLE001
        return getattr(ex, "status", -1), b""


def _corrupt(data, rng):
    data = bytearray(data)
    for _ in range(int(rng.integers(0, 12))):
        if data:
            data[int(rng.integers(0, len(data)))] = int(rng.integers(0, 256))
    if data and rng.random() < 0.5:
        i = int(rng.integers(0, len(data)))
        w = int(rng.integers(1, 9))
        data[i:i + w] = b"\xff" * len(data[i:i + w])
    if data and rng.random() < 0.5:
        data = data[:int(rng.integers(0, len(data)))]
    return bytes(data)


def test_mutated_and_garbage_streams_match_oracle(gpu, orc):
    """lib.rs:565-604: corrupted streams never fault; the result (bytes or
    error kind) equals the scalar reference's."""
    rng = np.random.default_rng(9)
    for _ in range(150):
        data = rng.integers(0, 40, int(rng.integers(0, 2000))).astype(np.uint8).tobytes()
        enc = orc.encode(data, int(rng.integers(0, 2)))
        bad = _corrupt(enc, rng)
        want = orc.decode_status(bad, max_len=len(data))
        got = _status(gpu.decode_bounded, bad, len(data))
        assert got == want
    for _ in range(100):
        g = bytearray(rng.integers(0, 256, int(rng.integers(0, 256))).astype(np.uint8).tobytes())
        for tag in (None, 0, 1):
            b = bytearray(g)
            if tag is not None:
                if b:
                    b[0] = tag
                else:
                    b.append(tag)
            want = orc.decode_status(bytes(b), max_len=1 << 16)
            assert _status(gpu.decode_bounded, bytes(b), 1 << 16) == want


def test_multiword_renorm_states(gpu, orc):
    """States below 2^16 in the header make a lane take several words per
    step (scalar.rs:233-235); the decoder must follow the scalar loop."""
    rng = np.random.default_rng(4)
    data = rng.integers(0, 6, 3000).astype(np.uint8).tobytes()
    for order in (0, 1):
        enc = bytearray(orc.encode(data, order))
        k = sum(bin(b).count("1") for b in enc[9:41])
        hdr = 9 + (512 if order == 0 else 32 + 512 * k)
        for lane in (0, 5, 31):
            e2 = bytearray(enc)
            e2[hdr + 4 * lane:hdr + 4 * lane + 4] = (0).to_bytes(4, "little")
            want = orc.decode_status(bytes(e2), max_len=len(data))
            assert _status(gpu.decode_bounded, bytes(e2), len(data)) == want


@pytest.mark.gpu
def test_plain_c_caller_round_trips(tmp_path):
    """The C ABI from a C99 program (no Python in between): both orders
    round-trip and the bounded decode rejects an inflated length."""
    import subprocess

    from test_capi_cpu import _build_c_caller

    r = subprocess.run([_build_c_caller(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "order 1:" in r.stdout
