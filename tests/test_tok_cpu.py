"""CPU checks of the read-name tokenizer row (crates/fqxv-tokenizer/src/lib.rs).

* The oracle (oracle/tokenizer_oracle.py) is pinned on the names payloads the
  reference stored in its golden archives: decode, re-encode, same bytes.
* The library's tokenizer host code (fqxv_b200/csrc/tok_capi.cu: role streams,
  op runs, byte planes, payload framing, error order) is compiled on its own
  with the two batch-coder calls it makes restated over the C oracle
  (oracle/tok_coder_stub.c, oracle/_build/libcallers_cpu.so), and checked against the oracle tokenizer on
  random blocks and on thousands of mutated payloads. The GPU coder itself is
  covered by tests/test_gpu_tok.py.
"""

import ctypes
import json
import os
import random
import subprocess

import numpy as np
import pytest

from conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden")
CODES = {"unsupported version": 48, "truncated": 49, "varint too long": 50,
         "record count exceeds token stream": 51, "op sym underrun": 52, "op run too long": 53,
         "op columns exceed the stream bound": 54, "delta plane length mismatch": 55,
         "MATCH without prior token": 56, "string data underrun": 57, "pad underrun": 58,
         "delta underrun": 59, "DELTA without numeric prior": 60, "unknown op": 61}


@pytest.fixture(scope="module")
def tok_oracle(orc):
    from oracle import tokenizer_oracle

    return tokenizer_oracle


@pytest.fixture(scope="module")
def golden_names():
    with open(os.path.join(GOLDEN, "fixture_names.json")) as f:
        idx = json.load(f)["payloads"]
    with open(os.path.join(GOLDEN, "fixture_names.bin"), "rb") as f:
        blob = f.read()
    return [blob[e["offset"]:e["offset"] + e["length"]] for e in idx if e["length"]]


@pytest.fixture(scope="module")
def tokcheck(orc):
    lib = os.path.join(ROOT, "oracle", "_build", "libcallers_cpu.so")
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), lib])
    L = ctypes.CDLL(lib)
    vp, sz = ctypes.c_void_p, ctypes.c_size_t
    u64p = ctypes.POINTER(ctypes.c_uint64)
    L.fqxv_tok_encode_host.argtypes = [vp, vp, vp, sz, vp, sz, vp, ctypes.c_uint64, vp, u64p]
    L.fqxv_tok_decode_host.argtypes = [vp, vp, vp, sz, vp, ctypes.c_uint64, vp, ctypes.c_uint64, vp, vp, u64p, u64p]
    return L


def _spans(lens):
    lens = np.asarray(lens, dtype=np.uint64)
    o = np.zeros(len(lens), np.uint64)
    if len(lens):
        o[1:] = np.cumsum(lens)[:-1]
    return np.ascontiguousarray(np.stack([o, lens], 1)) if len(lens) else np.zeros((1, 2), np.uint64)


def _encode(L, blocks):
    names = [bytes(n) for b in blocks for n in b]
    arena = np.frombuffer(b"".join(names) or b"\0", np.uint8).copy()
    nsp, bsp = _spans([len(n) for n in names]), _spans([len(b) for b in blocks])
    cap = 8 * arena.size + 100000 * len(blocks) + 4096
    dst = np.zeros(cap, np.uint8)
    out = np.zeros((max(1, len(blocks)), 2), np.uint64)
    need = ctypes.c_uint64()
    st = L.fqxv_tok_encode_host(1, arena.ctypes.data, nsp.ctypes.data, len(names), bsp.ctypes.data, len(blocks),
                                dst.ctypes.data, cap, out.ctypes.data, ctypes.byref(need))
    assert st == 0
    return [dst[int(o):int(o + n)].tobytes() for o, n in out[:len(blocks)]]


def _decode(L, payloads):
    arena = np.frombuffer(b"".join(payloads) or b"\0", np.uint8).copy()
    psp, n = _spans([len(p) for p in payloads]), len(payloads)
    ncap, scap = 64 * arena.size + 4096, 8 * arena.size + 64
    hn = np.zeros(ncap, np.uint8)
    nsp = np.zeros((scap, 2), np.uint64)
    bl = np.zeros((max(n, 1), 2), np.uint64)
    stt = np.zeros(max(n, 1), np.int32)
    a, b = ctypes.c_uint64(), ctypes.c_uint64()
    st = L.fqxv_tok_decode_host(1, arena.ctypes.data, psp.ctypes.data, n, hn.ctypes.data, ncap, nsp.ctypes.data,
                                scap, bl.ctypes.data, stt.ctypes.data, ctypes.byref(a), ctypes.byref(b))
    assert st != 17
    out = []
    for k in range(n):
        f, c = int(bl[k, 0]), int(bl[k, 1])
        out.append((int(stt[k]), [hn[int(o):int(o + l)].tobytes() for o, l in nsp[f:f + c]]))
    return out


def _oracle_decode(T, orc, p):
    try:
        return 0, T.decode(p)
    except T.TokError as e:
        return CODES[e.message], []
    except orc.OracleError as e:
        return e.status, []


def random_blocks(seed, n_blocks=30):
    rng = random.Random(seed)

    def name(i, style):
        if style == 0:
            return b"INST%d:41:HFXX:%d:%d:%d:%d" % (rng.randrange(9), rng.randrange(1, 3), 1101 + i // 50,
                                                   rng.randrange(30000), rng.randrange(30000))
        if style == 1:
            return b"read_%05d runid=x" % i
        if style == 2:
            return bytes(rng.choice(b"0123456789ab:_ ") for _ in range(rng.randrange(0, 30)))
        return b"SRR%d.%d %d length=%d" % (rng.randrange(10 ** rng.randrange(1, 20)), i, i, rng.randrange(300))

    blocks = []
    for _ in range(n_blocks):
        style = rng.randrange(4)
        blocks.append([name(i, style) for i in range(rng.randrange(0, 60))])
    blocks.append([b"0000123", b"0000124", b"99999999999999999999999", b"x" * 70 + b"1" * 5])
    return blocks


def mutate(rng, p):
    p = bytearray(p)
    k = rng.randrange(4)
    if k == 0:
        p[rng.randrange(len(p))] ^= 1 << rng.randrange(8)
    elif k == 1:
        p = p[:rng.randrange(len(p))]
    elif k == 2:
        p[rng.randrange(len(p))] = rng.randrange(256)
    else:
        i = rng.randrange(len(p))
        p[i:i] = bytes([rng.randrange(256)])
    return bytes(p)


def test_oracle_pinned_on_golden_payloads(tok_oracle, golden_names):
    assert len(golden_names) == 3
    for p in golden_names:
        names = tok_oracle.decode(p)
        assert names and tok_oracle.encode(names) == p


def test_oracle_roundtrip_and_reference_tests(tok_oracle):
    T = tok_oracle
    assert T.decode(T.encode([])) == []                      # lib.rs roundtrip_empty
    for blk in random_blocks(3, 10):
        if max((len(T.tokenize(n)) for n in blk), default=0) <= 64:
            assert T.decode(T.encode(blk)) == blk
    # lib.rs corrupt_run_length_cannot_drive_huge_allocation
    out = bytearray([1])
    T.write_varint(out, (1 << 64) // 4)
    counts = bytearray()
    T.write_varint(counts, 1)
    T.push_stream(out, counts)
    for _ in range(4):
        T.push_stream(out, b"")
    oc = bytearray()
    for c in range(64):
        T.write_varint(oc, 1 if c == 0 else 0)
    ol = bytearray()
    T.write_varint(ol, 1 << 30)
    for s in (oc, bytes([0]), ol):
        T.push_stream(out, s)
    with pytest.raises(T.TokError) as e:
        T.decode(bytes(out))
    assert e.value.message == "record count exceeds token stream"


def test_host_code_matches_oracle(tokcheck, tok_oracle, orc, golden_names):
    T = tok_oracle
    res = _decode(tokcheck, golden_names)
    assert all(st == 0 and names == T.decode(p) for (st, names), p in zip(res, golden_names))
    assert _encode(tokcheck, [T.decode(p) for p in golden_names]) == golden_names
    blocks = random_blocks(1)
    want = [T.encode(b) for b in blocks]
    assert _encode(tokcheck, blocks) == want
    for (st, names), w in zip(_decode(tokcheck, want), want):
        assert (st, names) == _oracle_decode(T, orc, w)


def test_host_code_error_order_matches_oracle(tokcheck, tok_oracle, orc, golden_names):
    T = tok_oracle
    rng = random.Random(5)
    pool = [T.encode(b) for b in random_blocks(2, 12)] + golden_names
    bad = [mutate(rng, rng.choice(pool)) for _ in range(1200)]
    got = _decode(tokcheck, bad)
    statuses = set()
    for (st, names), p in zip(got, bad):
        assert (st, names) == _oracle_decode(T, orc, p)
        statuses.add(st)
    assert len(statuses) >= 6


def edge_blocks():
    return [
        [b"", b"", b"a"],                                          # empty names
        [b"000", b"0", b"00", b"0000000000000000007", b"7"],       # zero padding, value 0
        [b"1234567890123456789", b"1234567890123456788"],          # 19 digits: a string token
        [b"x" + b"1" * 18, b"x" + b"1" * 17 + b"2"],               # 18 digits: numeric, delta
        [b":".join(b"%d" % k for k in range(80)), b":".join(b"%d" % (k + 1) for k in range(80))],  # > 64 tokens
        [b"A:1", b"A:1", b"A:1:2", b"A", b"A:3"],                  # token counts change between names
    ]


def test_host_code_edge_cases_match_oracle(tokcheck, tok_oracle, orc):
    T = tok_oracle
    blocks = edge_blocks()
    want = [T.encode(b) for b in blocks]
    assert _encode(tokcheck, blocks) == want
    for (st, names), w in zip(_decode(tokcheck, want), want):
        assert (st, names) == _oracle_decode(T, orc, w)
    # names of more than 64 tokens share the last column, which the
    # reference's decode rejects ("op run too long"); so does this one
    assert _decode(tokcheck, [want[4]])[0][0] == CODES["op run too long"]
