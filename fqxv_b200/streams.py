"""The coder's other container callers over the B200 coder
(include/fqxv_streams_gpu.h):

    put_stream(out, raw) / get_stream(src, pos)    fqxv-lroverlap codec.rs:289-363
    put_streams(raws) / get_streams(src, pos, n)   the same, batched in one GPU pass
    encode_perm(order) / decode_permutation(c, n)  fqxv reorder.rs:597-609, :1089-1105

Errors: `Corrupt` (fqxv_lroverlap::Error::Corrupt) and `PermError` with the
reference's Malformed text. No CPU fallback.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import rans


class Corrupt(rans.Error):
    """fqxv_lroverlap::Error::Corrupt: "malformed lroverlap block"."""


class PermError(rans.Error):
    """fqxv::Error::Malformed("bad permutation" | "permutation length mismatch")."""


def _ctx(device: int):
    from . import frame

    return frame.codec(device)._h


def put_streams(raws, device: int = 0) -> list[bytes]:
    """put_stream for each raw stream; every stream coded in one pass."""
    raws = [bytes(r) for r in raws]
    arena = np.frombuffer(b"".join(raws) or b"\0", dtype=np.uint8)
    lens = np.array([len(r) for r in raws], dtype=np.uint64)
    offs = np.zeros(len(raws), dtype=np.uint64)
    if len(raws):
        offs[1:] = np.cumsum(lens)[:-1]
    sp = np.ascontiguousarray(np.stack([offs, lens], 1)) if raws else np.zeros((1, 2), np.uint64)
    out = np.zeros((max(len(raws), 1), 2), dtype=np.uint64)
    need = ctypes.c_uint64(0)
    cap = int(lens.sum()) + 700 * len(raws) + 64
    dst = np.zeros(cap, dtype=np.uint8)
    st = rans.lib().fqxv_put_streams_host(_ctx(device), arena.ctypes.data, sp.ctypes.data, len(raws),
                                          dst.ctypes.data, cap, out.ctypes.data, ctypes.byref(need))
    rans.raise_for(st)
    return [dst[int(o):int(o + n)].tobytes() for o, n in out[:len(raws)]]


def put_stream(out: bytearray, raw, device: int = 0) -> None:
    out += put_streams([raw], device)[0]


def get_streams(src, pos: int, n: int, device: int = 0):
    """n streams read from src at pos: (streams, position after the last one).
    Raises Corrupt at the first failing one."""
    a = np.frombuffer(bytes(src) or b"\0", dtype=np.uint8)
    length = len(bytes(src))
    out = np.zeros((max(n, 1), 2), dtype=np.uint64)
    status = np.zeros(max(n, 1), dtype=np.int32)
    end, need = ctypes.c_uint64(0), ctypes.c_uint64(0)
    cap = 1 << 20
    for _ in range(2):
        dst = np.zeros(cap, dtype=np.uint8)
        st = rans.lib().fqxv_get_streams_host(_ctx(device), a.ctypes.data, length, pos, n, dst.ctypes.data, cap,
                                              out.ctypes.data, status.ctypes.data, ctypes.byref(end),
                                              ctypes.byref(need))
        if st == 17 and need.value > cap:
            cap = need.value
            continue
        break
    if st == 64:
        raise Corrupt(st, rans.status_message(st))
    rans.raise_for(st)
    return [dst[int(o):int(o + l)].tobytes() for o, l in out[:n]], int(end.value)


def get_stream(src, pos: int, device: int = 0):
    s, end = get_streams(src, pos, 1, device)
    return s[0], end


def encode_perm(order, device: int = 0) -> bytes:
    """reorder.rs:597-609: the permutation's four byte planes, coded on the GPU."""
    o = np.ascontiguousarray(np.asarray(order, dtype=np.uint32))
    cap = 649 + 8 * o.size + 64
    dst = np.zeros(cap, dtype=np.uint8)
    n = ctypes.c_uint64(0)
    rans.raise_for(rans.lib().fqxv_perm_encode_host(_ctx(device), o.ctypes.data, o.size, dst.ctypes.data, cap,
                                                    ctypes.byref(n)))
    return dst[:n.value].tobytes()


def decode_permutation(perm_c, n: int, device: int = 0) -> np.ndarray:
    """reorder.rs:1089-1105."""
    c = np.frombuffer(bytes(perm_c) or b"\0", dtype=np.uint8)
    out = np.zeros(max(n, 1), dtype=np.uint32)
    st = rans.lib().fqxv_perm_decode_host(_ctx(device), c.ctypes.data, len(bytes(perm_c)), n, out.ctypes.data)
    if st in (65, 66):
        raise PermError(st, rans.status_message(st))
    rans.raise_for(st)
    return out[:n]
