"""CPU restatement of the coder's other container callers -- TEST
INFRASTRUCTURE ONLY (the checker of include/fqxv_streams_gpu.h):

* put_stream / get_stream, crates/fqxv-lroverlap/src/codec.rs:289-363: a
  stream framed as [varint raw_len]([varint enc_len][rANS]), the smaller order
  with ties to order-1; any failure is Error::Corrupt;
* the reorder permutation, crates/fqxv/src/container/reorder.rs:597-609 and
  :1089-1105: n u32 as four byte planes coded as one stream, the smaller order
  with ties to order-0; decode bounded by 4 n.

Pinned by the nine put_stream streams of the reference's long-read fixture
(tests/golden/fixture_streams.*: the tile layout's lens ... literals streams):
re-framing their decoded bytes reproduces the stored streams.
"""

from __future__ import annotations

from . import oracle
from .tokenizer_oracle import Reader, TokError, write_varint


class Corrupt(Exception):
    pass


class PermError(Exception):
    def __init__(self, message: str):
        super().__init__(message)
        self.message = message


def put_stream(out: bytearray, raw: bytes) -> None:
    write_varint(out, len(raw))
    if not raw:
        return
    e0, e1 = oracle.encode(raw, 0), oracle.encode(raw, 1)
    enc = e1 if len(e1) <= len(e0) else e0
    write_varint(out, len(enc))
    out += enc


def get_stream(src: bytes, pos: int) -> tuple[bytes, int]:
    r = Reader(src)
    r.pos = pos
    try:
        raw_len = r.varint()
        if raw_len == 0:
            return b"", r.pos
        enc_len = r.varint()
        enc = r.take(enc_len)
    except TokError:
        raise Corrupt()
    st, out = oracle.decode_status(enc, max_len=raw_len)
    if st or len(out) != raw_len:
        raise Corrupt()
    return out, r.pos


def encode_perm(order) -> bytes:
    n = len(order)
    planes = bytearray(4 * n)
    for i, x in enumerate(order):
        for k in range(4):
            planes[k * n + i] = (x >> (8 * k)) & 0xFF
    o0, o1 = oracle.encode(bytes(planes), 0), oracle.encode(bytes(planes), 1)
    return o0 if len(o0) <= len(o1) else o1


def decode_permutation(perm_c: bytes, n: int) -> list[int]:
    st, pb = oracle.decode_status(perm_c, max_len=4 * n)
    if st:
        raise PermError("bad permutation")
    if len(pb) != 4 * n:
        raise PermError("permutation length mismatch")
    return [pb[i] | pb[n + i] << 8 | pb[2 * n + i] << 16 | pb[3 * n + i] << 24 for i in range(n)]
