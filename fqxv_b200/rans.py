"""Python front end of libfqxv_rans_gpu.so, shaped like the reference crate's
public API (crates/fqxv-rans/src/lib.rs:40-255):

    encode(src, Order.Zero | Order.One) -> bytes          lib.rs:111
    decode(src) -> bytes                                  lib.rs:186
    decode_bounded(src, max_len) -> bytes                 lib.rs:226
    decode_with(src, Backend.X) -> bytes                  lib.rs:241
    Backend.detect()                                      lib.rs:82

Errors are raised as `Malformed(message)` with the reference's message text
(`Error::Malformed(&'static str)`, lib.rs:42-52). Coding always runs on the
GPU; there is no CPU fallback, and a missing library or device raises.
"""

from __future__ import annotations

import ctypes
import enum
import os

from . import build as _build

_lib = None


class Order(enum.IntEnum):
    """lib.rs:59-64, plus the two keep-the-smaller rules of the callers."""
    Zero = 0
    One = 1
    BestTie0 = 2   # fqxv-tokenizer/src/lib.rs:91-95: ties keep order-0
    BestTie1 = 3   # fqxv-lroverlap/src/codec.rs:293-306: ties keep order-1


class Backend(enum.IntEnum):
    """lib.rs:68-77. All backends produce identical bytes; the GPU ignores it."""
    Scalar = 0
    Sse42 = 1
    Avx2 = 2
    Avx512 = 3

    @staticmethod
    def detect() -> "Backend":
        flags = ""
        try:
            with open("/proc/cpuinfo") as f:
                for line in f:
                    if line.startswith("flags"):
                        flags = line
                        break
        except OSError:
            pass
        toks = set(flags.split())
        if "avx512f" in toks:
            return Backend.Avx512
        if "avx2" in toks:
            return Backend.Avx2
        if "sse4_2" in toks:
            return Backend.Sse42
        return Backend.Scalar


class Error(Exception):
    """lib.rs:42-52."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status
        self.message = message


class Malformed(Error):
    """Error::Malformed: the stream was malformed or truncated."""


class DeviceError(Error):
    """No reference counterpart: a CUDA or API failure."""


MALFORMED = {1, 2, 3, 4, 5, 6, 7, 8}
# Statuses a batch call reports per stream (the call itself succeeded):
# the Malformed kinds and FQXV_RANS_E_TIMEOUT (a bounded device wait gave up).
TIMEOUT = 21
# The extended format's own failure (include/fqxv_rans_x_gpu.h), no
# reference counterpart.
X_MALFORMED = 9
STREAM_STATUSES = MALFORMED | {TIMEOUT, X_MALFORMED}


def lib_path() -> str:
    return _build.LIB


def lib() -> ctypes.CDLL:
    """Load the CUDA library (building it first when sources are newer)."""
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path) or not _build.up_to_date():
            try:
                _build.build()
            except Exception:
                if not os.path.exists(path):
                    raise
        L = ctypes.CDLL(path)
        u8p = ctypes.c_void_p
        sz = ctypes.c_size_t
        szp = ctypes.POINTER(ctypes.c_size_t)
        L.fqxv_rans_status_message.restype = ctypes.c_char_p
        L.fqxv_rans_status_message.argtypes = [ctypes.c_int]
        L.fqxv_rans_version.restype = ctypes.c_char_p
        L.fqxv_rans_encode_bound.restype = sz
        L.fqxv_rans_encode_bound.argtypes = [sz, ctypes.c_int]
        L.fqxv_rans_encode.argtypes = [u8p, sz, ctypes.c_int, u8p, sz, szp]
        L.fqxv_rans_peek_output_len.argtypes = [u8p, sz, ctypes.POINTER(ctypes.c_uint64)]
        L.fqxv_rans_decode.argtypes = [u8p, sz, u8p, sz, szp]
        L.fqxv_rans_decode_bounded.argtypes = [u8p, sz, sz, u8p, sz, szp]
        L.fqxv_rans_decode_with.argtypes = [u8p, sz, ctypes.c_int, u8p, sz, szp]
        L.fqxv_rans_ctx_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.fqxv_rans_ctx_destroy.argtypes = [ctypes.c_void_p]
        L.fqxv_rans_ctx_destroy.restype = None
        L.fqxv_rans_ctx_stream.argtypes = [ctypes.c_void_p]
        L.fqxv_rans_ctx_stream.restype = ctypes.c_void_p
        L.fqxv_rans_ctx_device_bytes.argtypes = [ctypes.c_void_p]
        L.fqxv_rans_ctx_device_bytes.restype = ctypes.c_uint64
        L.fqxv_rans_encode_batch_bound.argtypes = [u8p, sz, ctypes.c_int]
        L.fqxv_rans_encode_batch_bound.restype = ctypes.c_uint64
        L.fqxv_rans_encode_batch.argtypes = [ctypes.c_void_p, u8p, u8p, sz, ctypes.c_int, u8p, ctypes.c_uint64,
                                             u8p, u8p, ctypes.c_int]
        L.fqxv_rans_decode_batch.argtypes = [ctypes.c_void_p, u8p, u8p, sz, ctypes.c_uint64, u8p, u8p, u8p, u8p,
                                             ctypes.c_int]
        L.fqxv_rans_encode_batch_host.argtypes = [ctypes.c_void_p, u8p, u8p, sz, ctypes.c_int, u8p,
                                                  ctypes.c_uint64, u8p, u8p]
        L.fqxv_rans_decode_batch_host.argtypes = [ctypes.c_void_p, u8p, u8p, sz, ctypes.c_uint64, u8p, u8p, u8p,
                                                  u8p]
        # CRC-32C and block frames (include/fqxv_frame_gpu.h)
        vp = ctypes.c_void_p
        L.fqxv_crc32c_batch.argtypes = [vp, u8p, u8p, sz, u8p]
        L.fqxv_crc32c_batch_host.argtypes = [vp, u8p, u8p, sz, u8p]
        L.fqxv_crc32c_combine.restype = ctypes.c_uint32
        L.fqxv_crc32c_combine.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64]
        L.fqxv_frame_blocks_bound.restype = ctypes.c_uint64
        L.fqxv_frame_blocks_bound.argtypes = [u8p, sz, ctypes.c_int]
        L.fqxv_frame_blocks.argtypes = [vp, u8p, u8p, sz, ctypes.c_int, u8p, ctypes.c_uint64, u8p, u8p, u8p]
        L.fqxv_frame_blocks_host.argtypes = [vp, u8p, u8p, sz, ctypes.c_int, u8p, ctypes.c_uint64, u8p, u8p, u8p]
        for fn in ("fqxv_read_blocks", "fqxv_read_blocks_host"):
            getattr(L, fn).argtypes = [vp, u8p, ctypes.c_uint64, sz, u8p, u8p, u8p, szp,
                                       ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_int)]
        L.fqxv_payload_stream_locs.argtypes = [vp, u8p, u8p, sz, ctypes.c_uint64, u8p, u8p]
        # read-name tokenizer (include/fqxv_tok_gpu.h)
        L.fqxv_tok_encode_host.argtypes = [vp, u8p, u8p, sz, u8p, sz, u8p, ctypes.c_uint64, u8p,
                                           ctypes.POINTER(ctypes.c_uint64)]
        L.fqxv_tok_decode_host.argtypes = [vp, u8p, u8p, sz, u8p, ctypes.c_uint64, u8p, ctypes.c_uint64, u8p, u8p,
                                           ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
        # put_stream framing and the permutation planes (include/fqxv_streams_gpu.h)
        L.fqxv_put_streams_host.argtypes = [vp, u8p, u8p, sz, u8p, ctypes.c_uint64, u8p,
                                            ctypes.POINTER(ctypes.c_uint64)]
        L.fqxv_get_streams_host.argtypes = [vp, u8p, ctypes.c_uint64, ctypes.c_uint64, sz, u8p, ctypes.c_uint64,
                                            u8p, u8p, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
        L.fqxv_perm_encode_host.argtypes = [vp, u8p, ctypes.c_uint64, u8p, ctypes.c_uint64,
                                            ctypes.POINTER(ctypes.c_uint64)]
        L.fqxv_perm_decode_host.argtypes = [vp, u8p, ctypes.c_uint64, ctypes.c_uint64, u8p]
        L.fqxv_rans_ctx_set_profiling.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.fqxv_rans_ctx_stage_stats.argtypes = [ctypes.c_void_p, u8p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                                ctypes.c_int]
        _lib = L
    return _lib


def status_message(status: int) -> str:
    return lib().fqxv_rans_status_message(status).decode()


def raise_for(status: int) -> None:
    if status == 0:
        return
    msg = status_message(status)
    if status in MALFORMED:
        raise Malformed(status, msg)
    raise DeviceError(status, msg)


def _view(data):
    """(pointer, length, keepalive) of a bytes-like object."""
    if isinstance(data, (bytes, bytearray, memoryview)):
        b = bytes(data)
        return ctypes.cast(ctypes.c_char_p(b), ctypes.c_void_p), len(b), b
    import numpy as np

    a = np.ascontiguousarray(data, dtype=np.uint8)
    return ctypes.c_void_p(a.ctypes.data), a.size, a


def encode_bound(n: int, order: int) -> int:
    return lib().fqxv_rans_encode_bound(n, int(order))


def encode(src, order: Order = Order.Zero) -> bytes:
    """lib.rs:111 `encode(src, order)`; never fails on valid arguments."""
    p, n, keep = _view(src)
    cap = encode_bound(n, int(order))
    out = ctypes.create_string_buffer(max(cap, 1))
    ol = ctypes.c_size_t(0)
    raise_for(lib().fqxv_rans_encode(p, n, int(order), out, cap, ctypes.byref(ol)))
    del keep
    return out.raw[:ol.value]


def peek_output_len(src) -> int | None:
    """lib.rs:207: the header's declared length, or None when too short."""
    b = bytes(src[:9])
    return int.from_bytes(b[1:9], "little") if len(b) >= 9 else None


# Largest output the host front end allocates; a larger declared length fails
# like the reference's fallible reservation (model.rs:199-205).
ALLOC_LIMIT = 1 << 36


def decode_bounded(src, max_len: int) -> bytes:
    """lib.rs:226: rejects a declared length above max_len before decoding."""
    p, n_in, keep = _view(src)
    n = peek_output_len(src)
    if n is not None and n > max_len:
        raise_for(7)
    cap = n if (n is not None and n <= ALLOC_LIMIT) else 0
    out = ctypes.create_string_buffer(max(cap, 1))
    ol = ctypes.c_size_t(0)
    raise_for(lib().fqxv_rans_decode_bounded(p, n_in, min(max_len, (1 << 64) - 1), out, cap,
                                             ctypes.byref(ol)))
    del keep
    return out.raw[:ol.value]


def decode(src) -> bytes:
    """lib.rs:186 `decode(src)`."""
    return decode_bounded(src, (1 << 64) - 1)


def decode_with(src, backend: Backend) -> bytes:
    """lib.rs:241 `decode_with(src, backend)`."""
    del backend
    return decode(src)
