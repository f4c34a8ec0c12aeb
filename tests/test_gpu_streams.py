"""GPU parity of the put_stream framing and the permutation planes
(include/fqxv_streams_gpu.h) against the oracle (oracle/streams_oracle.py) and
the reference's stored put_stream streams."""

import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def S():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from fqxv_b200 import streams

    return streams


@pytest.fixture(scope="module")
def SO(orc):
    from oracle import streams_oracle

    return streams_oracle


def test_put_get_streams(S, SO, orc, golden):
    rng = random.Random(4)
    raws = [orc.decode(s) for e, s in golden if "seq_tile" in e["stream"]]
    stored = [s for e, s in golden if "seq_tile" in e["stream"]]
    raws += [b"", bytes(rng.randrange(5) for _ in range(50000)), b"z" * 100, bytes(range(256)) * 40]
    want = []
    for r in raws:
        out = bytearray()
        SO.put_stream(out, r)
        want.append(bytes(out))
    got = S.put_streams(raws)
    assert got == want
    assert all(g.endswith(s) for g, s in zip(got, stored))
    buf = b"xy" + b"".join(got)
    streams, end = S.get_streams(buf, 2, len(raws))
    assert streams == raws and end == len(buf)
    bad = bytearray(buf)
    bad[2 + sum(len(g) for g in got[:3]) + 12] ^= 0x20
    with pytest.raises(S.Corrupt):
        S.get_streams(bytes(bad), 2, len(raws))


def test_permutation(S, SO):
    rng = np.random.default_rng(6)
    for n in (0, 1, 5, 1000, 300000):
        order = rng.permutation(n).astype(np.uint32)
        c = S.encode_perm(order)
        assert c == SO.encode_perm([int(x) for x in order]) if n <= 1000 else len(c) > 0
        assert np.array_equal(S.decode_permutation(c, n), order)
        if n:
            with pytest.raises(S.PermError) as e:
                S.decode_permutation(c, n - 1)
            assert "bad permutation" in str(e.value)
            with pytest.raises(S.PermError) as e:
                S.decode_permutation(c, n + 1)
            assert "permutation length mismatch" in str(e.value)
    big = rng.permutation(300000).astype(np.uint32)
    c = S.encode_perm(big)
    from oracle import oracle

    planes = oracle.decode(c)
    assert planes == np.concatenate([(big >> (8 * k)).astype(np.uint8) for k in range(4)]).tobytes()
