"""Parity at the edges of the format's rules, GPU against the oracle:

* normalisation's negative-residual path (crates/fqxv-rans/src/model.rs:246-260):
  histograms whose floor frequencies overshoot 4096, so buckets are drained
  down to 1 and the next strictly-largest bucket is re-picked by lowest index;
  order-0 and order-1 (contexts with many rare successors);
* every order-1 decoder class and its neighbours: alphabets |D| on both sides of
  each class boundary (one-warp decoder, shared-memory tables, global tables);
* config 3's long-read quality blocks at full size (2,000 ONT-like reads in
  256 KiB - 8 MiB blocks), CPU-encoded then GPU-decoded, and GPU-encoded.
"""

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


def _dev(a):
    import torch

    return torch.from_numpy(np.array(a, dtype=np.uint8, copy=True)).to("cuda")


def _floor_sum(counts):
    tot = int(counts.sum())
    return sum(max(1, int(c) * 4096 // tot) for c in counts if c)


def _drain_order1_data(rng, contexts=8):
    """Bytes whose order-1 tables drain: for each of `contexts` context bytes,
    (context, successor) pairs in a shuffled order with the successors'
    counts 56 x 1000 plus many singletons (floor sum 4224: diff -128), the
    large counts tied so the re-pick's lowest-index rule decides."""
    ctx_bytes = rng.choice(np.arange(1, 256), contexts, replace=False).astype(np.uint8)
    succ = np.setdiff1d(np.arange(256), ctx_bytes).astype(np.uint8)
    pairs = []
    for j, a in enumerate(ctx_bytes):
        order = rng.permutation(succ)
        counts = np.ones(len(succ), dtype=np.int64)
        counts[:56] = 1000 + (0 if j % 2 == 0 else rng.integers(0, 3, 56))
        s = np.repeat(order, counts)
        pairs.append(np.stack([np.full(len(s), a, dtype=np.uint8), s], 1))
    pairs = np.concatenate(pairs)
    pairs = pairs[rng.permutation(len(pairs))]
    return pairs.reshape(-1), ctx_bytes


def _order1_hist(data, ctx):
    prev = np.concatenate([[0], data[:-1]])
    return np.bincount(data[prev == ctx], minlength=256)


def test_negative_residual_order0(codec, orc):
    rng = np.random.default_rng(3)
    counts = np.ones(256, dtype=np.int64)
    counts[:56] = 10_000                          # 56 x 73 + 200 = 4288: diff = -192
    data = np.repeat(np.arange(256, dtype=np.uint8), counts)[rng.permutation(int(counts.sum()))]
    assert _floor_sum(np.bincount(data, minlength=256)) > 4096
    more = [data]
    for _ in range(6):                            # ties broken differently, other overshoots
        c = np.zeros(256, dtype=np.int64)
        idx = rng.permutation(256)
        nb = int(rng.integers(2, 30))
        c[idx[:nb]] = int(rng.integers(800, 20_000))
        c[idx[nb:nb + 180]] = 1
        d = np.repeat(np.arange(256, dtype=np.uint8), c)[rng.permutation(int(c.sum()))]
        assert _floor_sum(np.bincount(d, minlength=256)) > 4096
        more.append(d)
    for d in more:
        blob = d.tobytes()
        want = orc.encode(blob, 0)
        assert rans.encode(blob, rans.Order.Zero) == want
        assert rans.decode(want) == blob


def test_negative_residual_order1(codec, orc):
    rng = np.random.default_rng(4)
    for rep in range(3):
        data, ctx_bytes = _drain_order1_data(rng)
        for a in ctx_bytes:
            assert _floor_sum(_order1_hist(data, a)) > 4096
        blob = data.tobytes()
        want = orc.encode(blob, 1)
        assert rans.encode(blob, rans.Order.One) == want
        assert rans.decode(want) == blob
        for mode in (rans.Order.BestTie0, rans.Order.BestTie1):
            e0, e1 = orc.encode(blob, 0), orc.encode(blob, 1)
            best = (e1 if len(e1) <= len(e0) else e0) if mode == rans.Order.BestTie1 else \
                (e1 if len(e1) < len(e0) else e0)
            assert rans.encode(blob, mode) == best


def _alphabet_data(rng, nd, with_zero, n=200_000):
    """n bytes drawn from an alphabet that makes |D| = nd exactly: context 0
    is present from the first position, so without byte 0 among the symbols
    nd - 1 symbols are drawn."""
    if with_zero:
        syms = np.concatenate([[0], rng.choice(np.arange(1, 256), nd - 1, replace=False)])
    else:
        syms = rng.choice(np.arange(1, 256), nd - 1, replace=False)
    # skewed so that normalisation rounds, with every symbol present after every context
    p = rng.dirichlet(np.full(len(syms), 0.7))
    p = 0.9 * p + 0.1 / len(syms)
    d = rng.choice(syms, n, p=p).astype(np.uint8)
    return d


def _dense_size(data):
    prev = np.concatenate([[0], data[:-1]])
    return len(set(np.unique(prev).tolist()) | set(np.unique(data).tolist()))


CLASS_EDGES = [2, 5, 9, 10, 11, 12, 15, 16, 17, 24, 30, 31, 32, 33, 41, 46, 47, 48, 49, 64, 100, 256]


@pytest.mark.parametrize("nd", CLASS_EDGES)
def test_order1_decoder_class_edges(codec, orc, nd):
    rng = np.random.default_rng(1000 + nd)
    for with_zero in (False, True):
        if nd == 256 and not with_zero:
            continue
        data = _alphabet_data(rng, nd, with_zero)
        assert _dense_size(data) == nd
        blob = data.tobytes()
        want = orc.encode(blob, 1)
        assert rans.encode(blob, rans.Order.One) == want
        # decode through the batch path with per-stage launch counts, so the
        # class that decoded it is known
        codec.stage_stats(reset=True)
        d_out, lens, st = codec.decode_batch(_dev(np.frombuffer(want, np.uint8)), [[0, len(want)]],
                                             [[0, len(blob)]])
        assert (st == 0).all() and int(lens[0]) == len(blob)
        assert d_out[:len(blob)].cpu().numpy().tobytes() == blob
        used = {k for k, v in codec.stage_stats(reset=True).items() if v["launches"] and k.startswith("dec_o1")}
        assert len(used) == 1, used


def test_ont_blocks_full_size(codec, orc):
    data, spans = W.config3_ont()
    assert len(spans) >= 2 and int(spans[:, 1].max()) > (4 << 20)
    enc, eoff, elen = orc.encode_batch(data, spans[:, 0], spans[:, 1], 1)
    cs = np.stack([eoff, elen], axis=1)
    d_enc = _dev(enc)
    d_dec, lens, st = codec.decode_batch(d_enc, cs, spans)
    assert (st == 0).all() and (lens == spans[:, 1]).all()
    assert np.array_equal(d_dec[:len(data)].cpu().numpy(), data)
    d_out, out_spans, _ = codec.encode_batch(_dev(data), spans, 1)
    out = d_out.cpu().numpy()
    for i in range(len(spans)):
        got = out[int(out_spans[i, 0]):int(out_spans[i, 0] + out_spans[i, 1])]
        assert np.array_equal(got, enc[int(eoff[i]):int(eoff[i] + elen[i])]), i
