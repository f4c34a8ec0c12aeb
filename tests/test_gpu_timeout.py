"""Bounded device waits. A decode kernel stages each stream's tables into
shared memory with one bulk copy and waits on its mbarrier for a bounded
number of polls. When that wait gives up, the kernel drains the same copy
(so nothing lands in shared memory after the CTA moves on), reports
FQXV_RANS_E_TIMEOUT for the stream and keeps the context usable.

The give-up is forced with the test-only poll count of
include/fqxv_rans_gpu_testing.h (0 polls on the first wait), not by a fault:
every copy still lands and every drain succeeds."""

import numpy as np
import pytest

from fqxv_b200 import rans
from fqxv_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _batch(orc):
    """Streams of every decode class: order-0, order-1 with a small alphabet
    (one-warp decoder), order-1 full-range quality (shared-memory tables) and
    order-1 over 200 symbols (tables in global memory, no staged copy)."""
    rng = np.random.default_rng(5)
    blocks = [
        (W.binned_quality(70_000, seed=1).tobytes(), 0),
        (W.binned_quality(90_000, seed=2).tobytes(), 1),
        (W.full_quality(120_000, seed=3).tobytes(), 1),
        (W.full_quality(33_000, seed=4).tobytes(), 0),
        (rng.integers(0, 200, 50_000, dtype=np.uint8).tobytes(), 1),
    ]
    enc = [orc.encode(b, o) for b, o in blocks]
    arena = np.frombuffer(b"".join(enc), dtype=np.uint8).copy()
    lens = np.array([len(e) for e in enc], dtype=np.uint64)
    offs = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.uint64)
    raw = [b for b, _ in blocks]
    rl = np.array([len(b) for b in raw], dtype=np.uint64)
    ro = np.concatenate([[0], np.cumsum(rl)[:-1]]).astype(np.uint64)
    return arena, np.stack([offs, lens], 1), raw, np.stack([ro, rl], 1)


def test_first_wait_gives_up_then_recovers(orc):
    import torch

    from fqxv_b200.batch import Codec

    arena, spans, raw, out_spans = _batch(orc)
    staged = np.array([True, True, True, True, False])
    c = Codec(0)
    try:
        d_src = torch.from_numpy(arena).cuda()
        c._test_set_wait_polls(0)
        d_dst, lens, st = c.decode_batch(d_src, spans, out_spans, raise_on_error=False)
        torch.cuda.synchronize()
        assert (st[staged] == rans.TIMEOUT).all(), st
        assert (lens[staged] == 0).all()
        # the global-table decoder stages nothing and is unaffected
        assert (st[~staged] == 0).all(), st
        out = d_dst.cpu().numpy()
        for i in np.nonzero(~staged)[0]:
            o, n = int(out_spans[i, 0]), int(out_spans[i, 1])
            assert out[o:o + n].tobytes() == raw[i]
        # the same context decodes the batch correctly once the waits are bounded normally
        c._test_set_wait_polls(1 << 22)
        d_dst, lens, st = c.decode_batch(d_src, spans, out_spans)
        torch.cuda.synchronize()
        assert (st == 0).all() and (lens == out_spans[:, 1]).all()
        out = d_dst.cpu().numpy()
        for i in range(len(raw)):
            o, n = int(out_spans[i, 0]), int(out_spans[i, 1])
            assert out[o:o + n].tobytes() == raw[i], i
    finally:
        c.close()


def test_knob_reaches_every_stream_of_a_large_batch(orc):
    """More streams than CTAs: every CTA gives up on each stream it takes, so
    each of them must still carry a status (none left as a stale OK)."""
    import torch

    from fqxv_b200.batch import Codec

    blobs = [W.binned_quality(4096 + 97 * i, seed=i).tobytes() for i in range(600)]
    enc = [orc.encode(b, i % 2) for i, b in enumerate(blobs)]
    arena = np.frombuffer(b"".join(enc), dtype=np.uint8).copy()
    lens = np.array([len(e) for e in enc], dtype=np.uint64)
    offs = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.uint64)
    rl = np.array([len(b) for b in blobs], dtype=np.uint64)
    ro = np.concatenate([[0], np.cumsum(rl)[:-1]]).astype(np.uint64)
    c = Codec(0)
    try:
        d_src = torch.from_numpy(arena).cuda()
        c._test_set_wait_polls(0)
        _, _, st = c.decode_batch(d_src, np.stack([offs, lens], 1), np.stack([ro, rl], 1), raise_on_error=False)
        assert (st == rans.TIMEOUT).all()
        c._test_set_wait_polls(1 << 22)
        d_dst, _, st = c.decode_batch(d_src, np.stack([offs, lens], 1), np.stack([ro, rl], 1))
        assert (st == 0).all()
        assert d_dst[:int(rl.sum())].cpu().numpy().tobytes() == b"".join(blobs)
    finally:
        c.close()
