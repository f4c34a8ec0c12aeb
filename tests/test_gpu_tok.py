"""GPU parity of the read-name tokenizer (fqxv_b200.tokenizer over
libfqxv_rans_gpu.so) against the oracle restatement of
crates/fqxv-tokenizer/src/lib.rs and the names payloads the reference stored
in its golden archives. Byte work: payloads, names and statuses identical."""

import random

import numpy as np
import pytest

from test_tok_cpu import CODES, _oracle_decode, edge_blocks, mutate, random_blocks  # noqa: F401

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tok():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from fqxv_b200 import tokenizer

    return tokenizer


@pytest.fixture(scope="module")
def T(orc):
    from oracle import tokenizer_oracle

    return tokenizer_oracle


@pytest.fixture(scope="module")
def golden_names():
    import json
    import os

    from conftest import ROOT

    g = os.path.join(ROOT, "tests", "golden")
    idx = json.load(open(os.path.join(g, "fixture_names.json")))["payloads"]
    blob = open(os.path.join(g, "fixture_names.bin"), "rb").read()
    return [blob[e["offset"]:e["offset"] + e["length"]] for e in idx if e["length"]]


def test_golden_payloads(tok, T, golden_names):
    names = tok.decode_blocks(golden_names)
    assert names == [T.decode(p) for p in golden_names]
    assert tok.encode_blocks(names) == golden_names
    assert tok.encode(names[0]) == golden_names[0] and tok.decode(golden_names[1]) == names[1]


def test_random_blocks_match_oracle(tok, T, orc):
    blocks = random_blocks(11, 40)
    want = [T.encode(b) for b in blocks]
    assert tok.encode_blocks(blocks) == want
    got, st = tok.decode_blocks(want, raise_on_error=False)
    for g, s, w in zip(got, st, want):
        assert (int(s), g) == _oracle_decode(T, orc, w)
    assert tok.encode([]) == T.encode([]) and tok.decode(T.encode([])) == []


def test_mutated_payloads_match_oracle(tok, T, orc, golden_names):
    rng = random.Random(8)
    pool = [T.encode(b) for b in random_blocks(4, 10)] + golden_names
    bad = [mutate(rng, rng.choice(pool)) for _ in range(600)]
    got, st = tok.decode_blocks(bad, raise_on_error=False)
    seen = set()
    for g, s, p in zip(got, st, bad):
        assert (int(s), g) == _oracle_decode(T, orc, p)
        seen.add(int(s))
    assert len(seen) >= 6
    with pytest.raises(tok.Malformed) as e:
        tok.decode(b"\x02" + golden_names[0][1:])
    assert str(e.value) == "malformed name stream: unsupported version"


def test_large_batch_round_trip(tok, T):
    """200 blocks x 2000 Illumina-style names: one GPU pass each way; a few
    blocks against the oracle, every block round-tripped."""
    rng = np.random.default_rng(3)
    blocks = []
    for b in range(200):
        x = rng.integers(1000, 30000, 2000)
        y = rng.integers(1000, 30000, 2000)
        tile = 1101 + np.arange(2000) // 400
        blocks.append([b"A00123:8:H7KJ2DSXX:%d:%d:%d:%d" % (1 + b % 4, tile[i], x[i], y[i]) for i in range(2000)])
    payloads = tok.encode_blocks(blocks)
    for k in (0, 77, 199):
        assert payloads[k] == T.encode(blocks[k])
    assert tok.decode_blocks(payloads) == blocks


def test_edge_cases_match_oracle(tok, T, orc):
    blocks = edge_blocks()
    want = [T.encode(b) for b in blocks]
    assert tok.encode_blocks(blocks) == want
    got, st = tok.decode_blocks(want, raise_on_error=False)
    for g, s, w in zip(got, st, want):
        assert (int(s), g) == _oracle_decode(T, orc, w)
    assert int(st[4]) == CODES["op run too long"]
