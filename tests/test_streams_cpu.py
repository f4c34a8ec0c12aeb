"""CPU checks of the put_stream / get_stream framing (crates/fqxv-lroverlap/
src/codec.rs:289-363) and the permutation planes (crates/fqxv/src/container/
reorder.rs:597-609, :1089-1105): the oracle pinned on the reference's stored
put_stream streams, and the library's framing host code (built without a GPU
over the CPU coder, oracle/_build/libcallers_cpu.so) against the oracle."""

import ctypes
import os
import random
import subprocess

import numpy as np
import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def SO(orc):
    from oracle import streams_oracle

    return streams_oracle


@pytest.fixture(scope="module")
def callers(orc):
    lib = os.path.join(ROOT, "oracle", "_build", "libcallers_cpu.so")
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), lib])
    L = ctypes.CDLL(lib)
    vp, sz, u64p = ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint64)
    L.fqxv_put_streams_host.argtypes = [vp, vp, vp, sz, vp, ctypes.c_uint64, vp, u64p]
    L.fqxv_get_streams_host.argtypes = [vp, vp, ctypes.c_uint64, ctypes.c_uint64, sz, vp, ctypes.c_uint64, vp, vp,
                                        u64p, u64p]
    return L


def tile_streams(golden):
    return [s for e, s in golden if "seq_tile" in e["stream"]]


def lib_put(L, raws):
    arena = np.frombuffer(b"".join(raws) or b"\0", np.uint8).copy()
    lens = np.array([len(r) for r in raws], np.uint64)
    offs = np.zeros(len(raws), np.uint64)
    if len(raws):
        offs[1:] = np.cumsum(lens)[:-1]
    sp = np.ascontiguousarray(np.stack([offs, lens], 1)) if raws else np.zeros((1, 2), np.uint64)
    cap = int(lens.sum()) + 700 * len(raws) + 64
    dst = np.zeros(cap, np.uint8)
    out = np.zeros((max(1, len(raws)), 2), np.uint64)
    need = ctypes.c_uint64()
    assert L.fqxv_put_streams_host(1, arena.ctypes.data, sp.ctypes.data, len(raws), dst.ctypes.data, cap,
                                   out.ctypes.data, ctypes.byref(need)) == 0
    return [dst[int(o):int(o + n)].tobytes() for o, n in out[:len(raws)]]


def lib_get(L, buf, pos, n):
    a = np.frombuffer(buf or b"\0", np.uint8).copy()
    cap = 8 * len(buf) + (1 << 16)
    dst = np.zeros(cap, np.uint8)
    out = np.zeros((max(n, 1), 2), np.uint64)
    st = np.zeros(max(n, 1), np.int32)
    end, need = ctypes.c_uint64(), ctypes.c_uint64()
    r = L.fqxv_get_streams_host(1, a.ctypes.data, len(buf), pos, n, dst.ctypes.data, cap, out.ctypes.data,
                                st.ctypes.data, ctypes.byref(end), ctypes.byref(need))
    assert r != 17
    return r, [dst[int(o):int(o + l)].tobytes() for o, l in out[:n]], list(st[:n])


def oracle_get(SO, buf, pos, n):
    outs = []
    for _ in range(n):
        try:
            s, pos = SO.get_stream(buf, pos)
        except SO.Corrupt:
            return 64, outs
        outs.append(s)
    return 0, outs


def test_oracle_pinned_on_stored_put_streams(SO, orc, golden):
    streams = tile_streams(golden)
    assert len(streams) == 9
    for s in streams:
        raw = orc.decode(s)
        out = bytearray()
        SO.put_stream(out, raw)
        frame = bytearray()
        SO.write_varint(frame, len(raw))
        SO.write_varint(frame, len(s))
        assert bytes(out) == bytes(frame) + s      # the stored stream, re-framed exactly
        assert SO.get_stream(bytes(out), 0) == (raw, len(out))


def test_oracle_permutation(SO):
    rng = random.Random(1)
    for n in (0, 1, 7, 300):
        order = list(range(n))
        rng.shuffle(order)
        c = SO.encode_perm(order)
        assert SO.decode_permutation(c, n) == order
        if n:
            with pytest.raises(SO.PermError) as e:
                SO.decode_permutation(c, n - 1)
            assert e.value.message == "bad permutation"
            with pytest.raises(SO.PermError) as e:
                SO.decode_permutation(c, n + 1)
            assert e.value.message == "permutation length mismatch"


def test_host_framing_matches_oracle(SO, orc, callers, golden):
    rng = random.Random(2)
    raws = [orc.decode(s) for s in tile_streams(golden)]
    raws += [b"", bytes(rng.randrange(4) for _ in range(3000)), b"\x07" * 500, b"", bytes(range(256)) * 3]
    want = []
    for r in raws:
        out = bytearray()
        SO.put_stream(out, r)
        want.append(bytes(out))
    assert lib_put(callers, raws) == want
    buf = b"prefix" + b"".join(want) + b"tail"
    r, got, st = lib_get(callers, buf, 6, len(raws))
    assert r == 0 and got == raws and all(s == 0 for s in st)
    # mutations: the first failure and every stream before it agree
    for it in range(400):
        b = bytearray(buf)
        k = rng.randrange(3)
        i = rng.randrange(6, len(b) - 4)
        if k == 0:
            b[i] ^= 1 << rng.randrange(8)
        elif k == 1:
            b = b[:i]
        else:
            b[i] = rng.randrange(256)
        b = bytes(b)
        ost, ogot = oracle_get(SO, b, 6, len(raws))
        r, got, st = lib_get(callers, b, 6, len(raws))
        assert r == ost
        k_ok = len(ogot) if ost else len(raws)
        assert got[:k_ok] == ogot[:k_ok] and all(s == 0 for s in st[:k_ok])
        assert all(s == 64 for s in st[k_ok:])


def test_host_framing_edges(SO, callers):
    # no frames; a buffer that ends exactly after the last frame; a zero-length
    # frame; a truncated length varint
    assert lib_get(callers, b"abc", 3, 0) == (0, [], [])
    frames = lib_put(callers, [b"", b"q" * 40])
    buf = b"".join(frames)
    assert lib_get(callers, buf, 0, 2) == (0, [b"", b"q" * 40], [0, 0])
    r, got, st = lib_get(callers, buf, 0, 3)
    assert r == 64 and st == [0, 0, 64]
    r, got, st = lib_get(callers, b"\x80", 0, 1)
    assert r == 64 and st == [64]
