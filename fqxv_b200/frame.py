"""CRC-32C and container block frames on the GPU, shaped like the reference:

    crc32c(data) -> int                          crates/fqxv/src/crc.rs:74
    crc32c_combine(crc_a, crc_b, len_b) -> int   crc.rs:116
    write_blocks(payloads, terminate) -> bytes   crates/fqxv/src/container/block.rs:110-142
    read_block(buf, pos, index)                  block.rs:1209-1254
    read_blocks(buf) -> list[bytes]              read_block until the terminator
    payload_stream_locs(payload, block_offset)   block.rs:961-980

Errors follow crates/fqxv/src/lib.rs:167-178: `Truncated`, `Corrupt` (with
the reference's `what`, e.g. "block 3" or "block 3 (bad sync marker)") and
`Malformed`. Checksums and copies run on the GPU through
libfqxv_rans_gpu.so (one context per device, created on first use); there is
no CPU fallback. The batched forms are methods of `batch.Codec`.
"""

from __future__ import annotations

import threading

import numpy as np

from . import batch, rans

MAX_BLOCK_PAYLOAD = 1 << 31   # format.rs:87
FRAME_HEAD_LEN = 16           # format.rs:99

TRUNCATED, CORRUPT, BAD_SYNC, TOO_LARGE = 32, 33, 34, 35


class FrameError(Exception):
    """A container-level error (lib.rs:167-178)."""

    def __init__(self, status: int, message: str, index: int | None = None):
        super().__init__(message)
        self.status = status
        self.index = index


class Truncated(FrameError):
    """Error::Truncated: "truncated fqxv stream"."""


class Corrupt(FrameError):
    """Error::Corrupt { what }: "corrupted fqxv data: {what} (crc mismatch)"."""

    def __init__(self, status: int, what: str, index: int | None = None):
        super().__init__(status, "corrupted fqxv data: %s (crc mismatch)" % what, index)
        self.what = what


class Malformed(FrameError):
    """Error::Malformed(msg): "malformed fqxv block: {msg}"."""


def error_for(status: int, index: int) -> FrameError:
    if status == TRUNCATED:
        return Truncated(status, "truncated fqxv stream", index)
    if status == CORRUPT:
        return Corrupt(status, "block %d" % index, index)
    if status == BAD_SYNC:
        return Corrupt(status, "block %d (bad sync marker)" % index, index)
    if status == TOO_LARGE:
        return Malformed(status, "malformed fqxv block: block payload length exceeds the maximum", index)
    return FrameError(status, rans.status_message(status), index)


_codecs: dict[int, batch.Codec] = {}
_lock = threading.Lock()


def codec(device: int = 0) -> batch.Codec:
    """The module's context on `device` (created on first use)."""
    with _lock:
        c = _codecs.get(device)
        if c is None:
            c = _codecs[device] = batch.Codec(device)
        return c


def _host(data) -> np.ndarray:
    if isinstance(data, np.ndarray):
        return np.ascontiguousarray(data, dtype=np.uint8).reshape(-1)
    return np.frombuffer(bytes(data), dtype=np.uint8)


def crc32c(data, device: int = 0) -> int:
    """crc.rs:74: CRC-32C (Castagnoli, init and xor-out 0xFFFFFFFF)."""
    a = _host(data)
    n = a.size
    if n == 0:
        a = np.zeros(1, dtype=np.uint8)
    return int(codec(device).crc32c_batch_host(a, [(0, n)])[0])


def crc32c_combine(crc_a: int, crc_b: int, len_b: int) -> int:
    """crc.rs:116: crc32c(A ++ B) from crc32c(A), crc32c(B) and len(B)."""
    return int(rans.lib().fqxv_crc32c_combine(crc_a & 0xFFFFFFFF, crc_b & 0xFFFFFFFF, int(len_b)))


def write_blocks(payloads, terminate: bool = False, device: int = 0) -> bytes:
    """block.rs:110-142: [FQXB][u64 len][u32 crc32c][payload] per payload,
    back to back; `terminate` appends the zero-length terminator frame."""
    parts = [_host(p) for p in payloads]
    sizes = [p.size for p in parts]
    src = np.concatenate(parts) if parts and sum(sizes) else np.zeros(1, dtype=np.uint8)
    offs = np.concatenate([[0], np.cumsum(sizes)[:-1]]) if parts else np.zeros(0)
    spans = np.stack([offs, sizes], axis=1) if parts else np.zeros((0, 2))
    c = codec(device)
    need = c.frame_bound(spans, terminate)
    dst = np.zeros(max(need, 1), dtype=np.uint8)
    c.frame_blocks_host(src, spans, dst, terminate)
    return dst[:need].tobytes()


def read_blocks(buf, device: int = 0) -> list[bytes]:
    """Every block payload up to the terminator or a clean end, each CRC-checked
    (block.rs:1209-1254 in a loop); raises the first frame's error."""
    a = _host(buf)
    if a.size == 0:
        return []
    pay, _crcs, status, _consumed, _term = codec(device).read_blocks_host(a)
    out = []
    for k, (sp, st) in enumerate(zip(pay, status)):
        if st:
            raise error_for(int(st), k)
        out.append(a[int(sp[0]):int(sp[0] + sp[1])].tobytes())
    return out


def read_block(buf, pos: int = 0, index: int = 0, device: int = 0):
    """block.rs:1209: the payload of the frame at `pos` and the position after
    it, or None at the terminator or a clean end."""
    a = _host(buf)[pos:]
    if a.size < 4:
        return None
    pay, _crcs, status, consumed, term = codec(device).read_blocks_host(a, max_frames=1)
    if len(status) == 0:
        return None
    if status[0]:
        raise error_for(int(status[0]), index)
    off, ln = int(pay[0][0]), int(pay[0][1])
    return a[off:off + ln].tobytes(), pos + consumed


def payload_stream_locs(payload, block_offset: int, device: int = 0) -> list[tuple[int, int, int]]:
    """block.rs:961-980: (offset, len, crc32c) of the names, sequence and
    quality streams of a plain payload framed at `block_offset`."""
    import torch

    a = _host(payload)
    d = torch.from_numpy(a.copy() if a.size else np.zeros(1, dtype=np.uint8)).to("cuda:%d" % device)
    locs, status = codec(device).payload_stream_locs(d, [(0, a.size)], base=block_offset + FRAME_HEAD_LEN)
    if status[0]:
        raise error_for(int(status[0]), 0)
    return [(int(l["offset"]), int(l["len"]), int(l["crc"])) for l in locs[0]]
