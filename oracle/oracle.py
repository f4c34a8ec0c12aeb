"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

The oracle restates `crates/fqxv-rans` (model.rs, scalar.rs, lib.rs and the
order-0 SIMD backends avx2.rs / avx512.rs) in C (rans_oracle.c, rans_simd.c).
Only `tests/`, `__graft_entry__.smoke()` and `bench.py`'s CPU-baseline leg use
it, as the checker and as the timed CPU path; the product library never calls
it.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liborc_rans.so")

# Same numbering as include/fqxv_rans_gpu.h (messages: the reference's).
MESSAGES = {
    1: "truncated stream",
    2: "unknown order tag",
    3: "rANS freq table exceeds TOTFREQ",
    4: "rANS freq table does not sum to TOTFREQ",
    5: "symbol references absent context",
    6: "rANS output length too large to allocate",
    7: "rANS output length exceeds caller bound",
    8: "truncated renorm stream",
    9: "malformed extended stream",
    16: "invalid argument",
    17: "destination buffer too small",
    32: "truncated fqxv stream",
    33: "corrupted fqxv data: block (crc mismatch)",
    34: "corrupted fqxv data: block (bad sync marker) (crc mismatch)",
    35: "malformed fqxv block: block payload length exceeds the maximum",
}


class OracleError(Exception):
    def __init__(self, status: int):
        super().__init__("oracle status %d: %s" % (status, MESSAGES.get(status, "?")))
        self.status = status


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB_PATH):
        subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB_PATH


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        u8p = ctypes.POINTER(ctypes.c_uint8)
        sz = ctypes.c_size_t
        szp = ctypes.POINTER(ctypes.c_size_t)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        i32p = ctypes.POINTER(ctypes.c_int32)
        L.orc_encode_bound.restype = sz
        L.orc_encode_bound.argtypes = [sz, ctypes.c_int]
        for fn in ("orc_encode", "orc_encode_dispatch"):
            getattr(L, fn).argtypes = [u8p, sz, ctypes.c_int, u8p, sz, szp]
        for fn in ("orc_decode", "orc_decode_dispatch"):
            getattr(L, fn).argtypes = [u8p, sz, u8p, sz, szp]
        L.orc_decode_bounded.argtypes = [u8p, sz, sz, u8p, sz, szp]
        L.orc_encode_o0_simd.argtypes = [ctypes.c_int, u8p, sz, u8p, sz, szp]
        L.orc_decode_o0_simd.argtypes = [ctypes.c_int, u8p, sz, u8p, sz, szp]
        L.orc_simd_level.argtypes = []
        L.orc_normalize.argtypes = [ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint16)]
        L.orc_validate_freqs.argtypes = [ctypes.POINTER(ctypes.c_uint16)]
        L.orc_encsym_apply.restype = ctypes.c_uint32
        L.orc_encsym_apply.argtypes = [ctypes.c_uint32] * 3
        L.orc_magic_apply.restype = ctypes.c_uint32
        L.orc_magic_apply.argtypes = [ctypes.c_uint32] * 3
        L.orc_encode_batch.argtypes = [u8p, u64p, u64p, sz, ctypes.c_int, u8p, u64p, u64p, u64p, i32p,
                                       ctypes.c_int]
        L.orc_decode_batch.argtypes = [u8p, u64p, u64p, sz, u8p, u64p, u64p, u64p, i32p, ctypes.c_int]
        # CRC-32C and block frames (frame_oracle.c)
        L.orc_crc32c.restype = ctypes.c_uint32
        L.orc_crc32c.argtypes = [u8p, sz]
        L.orc_crc32c_update.restype = ctypes.c_uint32
        L.orc_crc32c_update.argtypes = [ctypes.c_uint32, u8p, sz]
        L.orc_crc32c_combine.restype = ctypes.c_uint32
        L.orc_crc32c_combine.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64]
        L.orc_frame_blocks.argtypes = [u8p, u64p, u64p, sz, ctypes.c_int, u8p, ctypes.c_uint64, u64p,
                                       ctypes.POINTER(ctypes.c_uint32), u64p]
        L.orc_read_blocks.argtypes = [u8p, ctypes.c_uint64, sz, u64p, u64p, ctypes.POINTER(ctypes.c_uint32), i32p,
                                      szp, u64p, ctypes.POINTER(ctypes.c_int)]
        L.orc_crc32c_batch.argtypes = [u8p, u64p, u64p, sz, ctypes.POINTER(ctypes.c_uint32), ctypes.c_int]
        L.orc_payload_stream_locs.argtypes = [u8p, ctypes.c_uint64, ctypes.c_uint64, u64p,
                                              ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)]
        _lib = L
    return _lib


def _buf(data) -> tuple[np.ndarray, ctypes.POINTER(ctypes.c_uint8)]:
    a = np.frombuffer(bytes(data), dtype=np.uint8) if not isinstance(data, np.ndarray) else data
    a = np.ascontiguousarray(a, dtype=np.uint8)
    if a.size == 0:
        a = np.zeros(1, dtype=np.uint8)[:0]
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))


def encode_bound(n: int, order: int) -> int:
    return lib().orc_encode_bound(n, order)


def encode(data, order: int, path: str = "scalar") -> bytes:
    """scalar.rs encode (path="scalar"), the reference's dispatch
    (path="dispatch"), or one SIMD level (path="avx2" / "avx512")."""
    a, p = _buf(data)
    cap = encode_bound(a.size, order)
    out = np.empty(cap, dtype=np.uint8)
    op = out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
    ol = ctypes.c_size_t(0)
    L = lib()
    if path == "scalar":
        st = L.orc_encode(p, a.size, order, op, cap, ctypes.byref(ol))
    elif path == "dispatch":
        st = L.orc_encode_dispatch(p, a.size, order, op, cap, ctypes.byref(ol))
    else:
        assert order == 0
        st = L.orc_encode_o0_simd({"avx2": 1, "avx512": 2}[path], p, a.size, op, cap, ctypes.byref(ol))
    if st:
        raise OracleError(st)
    return out[:ol.value].tobytes()


def peek_output_len(data) -> int | None:
    b = bytes(data[:9])
    return int.from_bytes(b[1:9], "little") if len(b) >= 9 else None


def decode(data, max_len: int | None = None, path: str = "scalar", cap: int | None = None) -> bytes:
    """scalar.rs decode. `cap` is the largest output the caller will allocate
    (a longer declared length fails with status 6, as `alloc_output` does);
    by default the declared length is allocated when it is under 1 GiB."""
    a, p = _buf(data)
    n = peek_output_len(a)
    if max_len is not None and n is not None and n > max_len:
        raise OracleError(7)
    if cap is None:
        cap = n if (n is not None and n <= (1 << 30)) else 0
    out = np.empty(max(cap, 1), dtype=np.uint8)
    op = out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
    ol = ctypes.c_size_t(0)
    L = lib()
    if path == "scalar":
        st = L.orc_decode(p, a.size, op, cap, ctypes.byref(ol))
    elif path == "dispatch":
        st = L.orc_decode_dispatch(p, a.size, op, cap, ctypes.byref(ol))
    else:
        st = L.orc_decode_o0_simd({"avx2": 1, "avx512": 2}[path], p, a.size, op, cap, ctypes.byref(ol))
    if st:
        raise OracleError(st)
    return out[:ol.value].tobytes()


def decode_status(data, max_len: int | None = None, cap: int | None = None) -> tuple[int, bytes]:
    try:
        return 0, decode(data, max_len=max_len, cap=cap)
    except OracleError as e:
        return e.status, b""


def normalize(counts) -> np.ndarray:
    c = np.ascontiguousarray(counts, dtype=np.uint32)
    f = np.zeros(256, dtype=np.uint16)
    lib().orc_normalize(c.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                        f.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)))
    return f


def validate_freqs(freq) -> int:
    f = np.ascontiguousarray(freq, dtype=np.uint16)
    return lib().orc_validate_freqs(f.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)))


def simd_level() -> int:
    return lib().orc_simd_level()


def _ptr(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def encode_batch(src: np.ndarray, offs: np.ndarray, lens: np.ndarray, order: int,
                 nthreads: int = 0) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Block-parallel encode over all host cores (order 2 = keep the smaller,
    ties to order 0). Returns (out arena, out offsets, out lengths)."""
    nb = len(offs)
    offs = np.ascontiguousarray(offs, dtype=np.uint64)
    lens = np.ascontiguousarray(lens, dtype=np.uint64)
    caps = np.array([encode_bound(int(l), 1 if order else 0) for l in lens], dtype=np.uint64)
    doff = np.zeros(nb, dtype=np.uint64)
    if nb:
        doff[1:] = np.cumsum(caps)[:-1]
    dst = np.empty(int(caps.sum()) if nb else 1, dtype=np.uint8)
    ol = np.zeros(nb, dtype=np.uint64)
    st = np.zeros(nb, dtype=np.int32)
    rc = lib().orc_encode_batch(_ptr(src, ctypes.c_uint8), _ptr(offs, ctypes.c_uint64), _ptr(lens, ctypes.c_uint64),
                                nb, order, _ptr(dst, ctypes.c_uint8), _ptr(doff, ctypes.c_uint64),
                                _ptr(caps, ctypes.c_uint64), _ptr(ol, ctypes.c_uint64), _ptr(st, ctypes.c_int32),
                                nthreads)
    if rc:
        raise OracleError(rc)
    return dst, doff, ol


def decode_batch(src: np.ndarray, offs: np.ndarray, lens: np.ndarray, out_lens: np.ndarray,
                 nthreads: int = 0) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    nb = len(offs)
    offs = np.ascontiguousarray(offs, dtype=np.uint64)
    lens = np.ascontiguousarray(lens, dtype=np.uint64)
    caps = np.ascontiguousarray(out_lens, dtype=np.uint64)
    doff = np.zeros(nb, dtype=np.uint64)
    if nb:
        doff[1:] = np.cumsum(caps)[:-1]
    dst = np.empty(max(int(caps.sum()), 1), dtype=np.uint8)
    ol = np.zeros(nb, dtype=np.uint64)
    st = np.zeros(nb, dtype=np.int32)
    rc = lib().orc_decode_batch(_ptr(src, ctypes.c_uint8), _ptr(offs, ctypes.c_uint64), _ptr(lens, ctypes.c_uint64),
                                nb, _ptr(dst, ctypes.c_uint8), _ptr(doff, ctypes.c_uint64),
                                _ptr(caps, ctypes.c_uint64), _ptr(ol, ctypes.c_uint64), _ptr(st, ctypes.c_int32),
                                nthreads)
    if rc:
        raise OracleError(rc)
    return dst, doff, ol


# ---- CRC-32C and block frames (frame_oracle.c) --------------------------------

def crc32c(data) -> int:
    """crates/fqxv/src/crc.rs:74."""
    a, p = _buf(data)
    return int(lib().orc_crc32c(p, a.size))


def crc32c_combine(crc_a: int, crc_b: int, len_b: int) -> int:
    """crc.rs:116."""
    return int(lib().orc_crc32c_combine(crc_a, crc_b, len_b))


def frame_blocks(src: np.ndarray, offs, lens, terminate: bool = False):
    """crates/fqxv/src/container/block.rs:110-142 over payloads of `src`.
    Returns (frames bytes, frame offsets, crcs)."""
    offs = np.ascontiguousarray(offs, dtype=np.uint64)
    lens = np.ascontiguousarray(lens, dtype=np.uint64)
    n = len(offs)
    need = int(lens.sum()) + 16 * n + (12 if terminate else 0)
    dst = np.zeros(max(need, 1), dtype=np.uint8)
    fo = np.zeros(max(n, 1), dtype=np.uint64)
    crcs = np.zeros(max(n, 1), dtype=np.uint32)
    tot = ctypes.c_uint64(0)
    src = np.ascontiguousarray(src, dtype=np.uint8)
    rc = lib().orc_frame_blocks(_ptr(src, ctypes.c_uint8), _ptr(offs, ctypes.c_uint64), _ptr(lens, ctypes.c_uint64),
                                n, 1 if terminate else 0, _ptr(dst, ctypes.c_uint8), need,
                                _ptr(fo, ctypes.c_uint64), _ptr(crcs, ctypes.c_uint32), ctypes.byref(tot))
    if rc:
        raise OracleError(rc)
    return dst[:need].tobytes(), fo[:n], crcs[:n]


def read_blocks(buf, max_frames: int | None = None):
    """block.rs:1209-1254 frame after frame. Returns (first status, payload
    spans (k, 2), crcs, status, consumed, terminated)."""
    a, p = _buf(buf)
    cap = a.size // 16 + 1 if max_frames is None else min(int(max_frames), a.size // 16 + 1)
    po = np.zeros(max(cap, 1), dtype=np.uint64)
    pl = np.zeros(max(cap, 1), dtype=np.uint64)
    crcs = np.zeros(max(cap, 1), dtype=np.uint32)
    st = np.zeros(max(cap, 1), dtype=np.int32)
    nf = ctypes.c_size_t(0)
    consumed = ctypes.c_uint64(0)
    term = ctypes.c_int(0)
    first = lib().orc_read_blocks(p, a.size, cap, _ptr(po, ctypes.c_uint64), _ptr(pl, ctypes.c_uint64),
                                  _ptr(crcs, ctypes.c_uint32), _ptr(st, ctypes.c_int32), ctypes.byref(nf),
                                  ctypes.byref(consumed), ctypes.byref(term))
    k = nf.value
    return first, np.stack([po[:k], pl[:k]], axis=1), crcs[:k], st[:k], consumed.value, bool(term.value)


def payload_stream_locs(payload, block_offset: int):
    """block.rs:961-980. Returns (status, [(offset, len, crc)] x 3)."""
    a, p = _buf(payload)
    off = np.zeros(3, dtype=np.uint64)
    ln = np.zeros(3, dtype=np.uint32)
    crc = np.zeros(3, dtype=np.uint32)
    rc = lib().orc_payload_stream_locs(p, a.size, block_offset, _ptr(off, ctypes.c_uint64),
                                       _ptr(ln, ctypes.c_uint32), _ptr(crc, ctypes.c_uint32))
    return rc, [(int(off[i]), int(ln[i]), int(crc[i])) for i in range(3)]


def crc32c_batch(src: np.ndarray, offs, lens, nthreads: int = 0) -> np.ndarray:
    """CRC-32C of many spans of `src` on host threads (the CPU baseline)."""
    offs = np.ascontiguousarray(offs, dtype=np.uint64)
    lens = np.ascontiguousarray(lens, dtype=np.uint64)
    out = np.zeros(max(len(offs), 1), dtype=np.uint32)
    src = np.ascontiguousarray(src, dtype=np.uint8)
    lib().orc_crc32c_batch(_ptr(src, ctypes.c_uint8), _ptr(offs, ctypes.c_uint64), _ptr(lens, ctypes.c_uint64),
                           len(offs), _ptr(out, ctypes.c_uint32), nthreads)
    return out[:len(offs)]

# --- extended stream format (rans_x.c): PARITY UNPINNED, test infrastructure


X_ORDER1, X_N4, X_STRIPE, X_RLE, X_PACK, X_CAT = 0x01, 0x02, 0x04, 0x08, 0x10, 0x20
X_MALFORMED = 9


def _x_lib():
    L = lib()
    if not getattr(L, "_x_ready", False):
        u8p = ctypes.POINTER(ctypes.c_uint8)
        sz = ctypes.c_size_t
        szp = ctypes.POINTER(ctypes.c_size_t)
        L.orc_x_encode_bound.restype = sz
        L.orc_x_encode_bound.argtypes = [sz, ctypes.c_int]
        L.orc_x_best_bound.restype = sz
        L.orc_x_best_bound.argtypes = [sz]
        L.orc_x_encode.argtypes = [u8p, sz, ctypes.c_int, u8p, sz, szp]
        L.orc_x_decode.argtypes = [u8p, sz, u8p, sz, szp]
        L.orc_x_encode_best.argtypes = [u8p, sz, u8p, sz, szp, ctypes.POINTER(ctypes.c_int)]
        L.orc_core_encode.argtypes = [u8p, sz, ctypes.c_int, ctypes.c_int, u8p, szp]
        L.orc_core_bound.restype = sz
        L.orc_core_bound.argtypes = [sz, ctypes.c_int, ctypes.c_int]
        L._x_ready = True
    return L


def x_encode(data, flags: int) -> bytes:
    """The extended stream of `data` with transform flags `flags`."""
    L = _x_lib()
    a, p = _buf(data)
    cap = L.orc_x_encode_bound(a.size, flags)
    out = np.empty(cap, dtype=np.uint8)
    n = ctypes.c_size_t(0)
    st = L.orc_x_encode(p, a.size, flags, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), cap, ctypes.byref(n))
    if st:
        raise OracleError(st)
    return out[:n.value].tobytes()


def x_encode_best(data) -> tuple[bytes, int]:
    """(stream, candidate index) of the selection over reference and
    extended candidates."""
    L = _x_lib()
    a, p = _buf(data)
    cap = L.orc_x_best_bound(a.size)
    out = np.empty(cap, dtype=np.uint8)
    n = ctypes.c_size_t(0)
    c = ctypes.c_int(0)
    st = L.orc_x_encode_best(p, a.size, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), cap, ctypes.byref(n),
                             ctypes.byref(c))
    if st:
        raise OracleError(st)
    return out[:n.value].tobytes(), c.value


def x_decode(stream, cap: int | None = None) -> bytes:
    """Decode an extended (or reference) stream; raises OracleError."""
    L = _x_lib()
    a, p = _buf(stream)
    if cap is None:
        cap = int.from_bytes(bytes(a[1:9]), "little") if a.size >= 9 else 0
    out = np.empty(max(cap, 1), dtype=np.uint8)
    n = ctypes.c_size_t(0)
    st = L.orc_x_decode(p, a.size, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), cap, ctypes.byref(n))
    if st:
        raise OracleError(st)
    return out[:n.value].tobytes()


def x_decode_status(stream, cap: int) -> int:
    L = _x_lib()
    a, p = _buf(stream)
    out = np.empty(max(cap, 1), dtype=np.uint8)
    n = ctypes.c_size_t(0)
    return L.orc_x_decode(p, a.size, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), cap, ctypes.byref(n))


def x_encode_batch(src: np.ndarray, offs, lens, flags: int, nthreads: int = 0):
    """Extended-format encode of every block on all host cores (flags 0x40:
    the selection). Returns (arena, offsets, lengths, choices)."""
    L = _x_lib()
    nb = len(offs)
    offs = np.ascontiguousarray(offs, dtype=np.uint64)
    lens = np.ascontiguousarray(lens, dtype=np.uint64)
    caps = np.array([L.orc_x_best_bound(int(n)) for n in lens], dtype=np.uint64)
    doff = np.zeros(nb, dtype=np.uint64)
    if nb:
        doff[1:] = np.cumsum(caps)[:-1]
    dst = np.empty(max(int(caps.sum()), 1), dtype=np.uint8)
    ol = np.zeros(nb, dtype=np.uint64)
    st = np.zeros(nb, dtype=np.int32)
    ch = np.zeros(nb, dtype=np.int32)
    L.orc_x_batch.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_size_t, ctypes.c_int, ctypes.c_int] + \
        [ctypes.c_void_p] * 6 + [ctypes.c_int]
    rc = L.orc_x_batch(src.ctypes.data, offs.ctypes.data, lens.ctypes.data, nb, flags, 0, dst.ctypes.data,
                       doff.ctypes.data, caps.ctypes.data, ol.ctypes.data, st.ctypes.data, ch.ctypes.data, nthreads)
    if rc:
        raise OracleError(rc)
    return dst, doff, ol, ch
