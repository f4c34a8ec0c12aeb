"""Serving runtime: requests submitted concurrently are coded in continuous
batches; every result equals the same request coded alone (single call) and
the oracle, and malformed requests fail with the reference's error kind
without disturbing the others in their batch."""

import threading

import numpy as np
import pytest

from fqxv_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from fqxv_b200 import rans, serve

    return rans, serve


def _requests(orc):
    rng = np.random.default_rng(12)
    reqs = []
    gens = list(W.GENERATORS.values())
    for i in range(36):
        n = int(np.exp(rng.uniform(np.log(1 << 10), np.log(1 << 20))))
        data = gens[i % 4](n, 100 + i).tobytes()
        if i % 3 == 0:
            reqs.append(("enc", data, int(rng.integers(0, 4))))
        else:
            order = int(rng.integers(0, 2))
            reqs.append(("dec", orc.encode(data, order), None))
    bad = bytearray(orc.encode(b"xyz" * 500, 1))
    reqs.append(("dec", bytes(bad[:60]), None))        # truncated
    bad[9 + 32] = 0xFF                                  # first table now exceeds TOTFREQ
    reqs.append(("dec", bytes(bad), None))
    return reqs


def _alone(rans, kind, data, order):
    try:
        return 0, (rans.encode(data, rans.Order(order)) if kind == "enc" else rans.decode(data))
    except rans.Malformed as e:
        return e.status, b""


def test_results_identical_alone_and_in_the_mix(gpu, orc):
    rans, serve = gpu
    reqs = _requests(orc)
    want = [_alone(rans, k, d, o) for k, d, o in reqs]
    # the single calls agree with the oracle
    for (k, d, o), (st, out) in zip(reqs, want):
        if k == "enc":
            e0, e1 = orc.encode(d, 0), orc.encode(d, 1)
            ref = {0: e0, 1: e1, 2: e1 if len(e1) < len(e0) else e0, 3: e1 if len(e1) <= len(e0) else e0}[o]
            assert out == ref
        else:
            assert (st, out) == orc.decode_status(d)
    got = [None] * len(reqs)
    with serve.Server(device=0, workers=3, hbm_cap=1 << 30) as srv:
        ids = [None] * len(reqs)

        def submitter(lo, hi):
            for i in range(lo, hi):
                k, d, o = reqs[i]
                ids[i] = srv.submit_encode(d, o) if k == "enc" else srv.submit_decode(d)

        ts = [threading.Thread(target=submitter, args=(a, min(a + 10, len(reqs)))) for a in range(0, len(reqs), 10)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        for i, rid in enumerate(ids):
            try:
                got[i] = (0, srv.result(rid))
            except rans.Malformed as e:
                got[i] = (e.status, b"")
        stats = srv.stats()
    assert got == want
    assert stats["completed"] == len(reqs)
    assert stats["batches"] < len(reqs), "requests were not batched together"


def test_admission_cap_serialises_but_completes(gpu, orc):
    rans, serve = gpu
    data = [W.full_quality(1 << 19, s).tobytes() for s in range(6)]
    with serve.Server(device=0, workers=2, hbm_cap=8 << 20) as srv:
        ids = [srv.submit_encode(d, rans.Order.One) for d in data]
        outs = [srv.result(i) for i in ids]
        with pytest.raises(rans.DeviceError):
            srv.submit_encode(bytes(64 << 20), rans.Order.One)   # larger than the cap
    for d, o in zip(data, outs):
        assert o == orc.encode(d, 1)


def test_bound_is_checked_at_submission(gpu, orc):
    rans, serve = gpu
    data = W.binned_quality(50_000, 3).tobytes()
    enc = orc.encode(data, 1)
    with serve.Server(device=0, workers=2, hbm_cap=1 << 30) as srv:
        bad = srv.submit_decode(enc, max_len=len(data) - 1)
        good = srv.submit_decode(enc, max_len=len(data))
        with pytest.raises(rans.Malformed) as e:
            srv.result(bad)
        assert e.value.status == 7
        assert srv.result(good) == data
