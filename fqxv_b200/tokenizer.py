"""Read-name tokenizer over the B200 coder, shaped like
`crates/fqxv-tokenizer/src/lib.rs`:

    encode(names) -> bytes          lib.rs:482
    decode(src) -> list[bytes]      lib.rs:543

plus the batched forms `encode_blocks` / `decode_blocks`, which code every
role stream of every block in one GPU pass (libfqxv_rans_gpu.so,
`fqxv_tok_encode_host` / `fqxv_tok_decode_host`). Payloads are byte-identical
to the reference's. Errors: `Malformed` with the reference's
"malformed name stream: ..." text, or `rans.Malformed` for a role stream's
rANS error. There is no CPU fallback.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import rans

TOK_STATUSES = set(range(48, 62))


class Malformed(rans.Error):
    """lib.rs:40-50 Error::Malformed."""


def _raise(status: int) -> None:
    if status in TOK_STATUSES:
        raise Malformed(status, rans.status_message(status))
    rans.raise_for(status)


def _codec(device: int):
    from . import frame

    return frame.codec(device)


def _spans(lens) -> np.ndarray:
    lens = np.asarray(lens, dtype=np.uint64)
    offs = np.zeros(len(lens), dtype=np.uint64)
    if len(lens):
        offs[1:] = np.cumsum(lens)[:-1]
    return np.ascontiguousarray(np.stack([offs, lens], axis=1)) if len(lens) else np.zeros((0, 2), np.uint64)


def encode_blocks(blocks, device: int = 0) -> list[bytes]:
    """One payload per block of names (each a list of bytes-like names)."""
    names = [bytes(n) for blk in blocks for n in blk]
    arena = np.frombuffer(b"".join(names) or b"\0", dtype=np.uint8)
    nsp = _spans([len(n) for n in names])
    counts = [len(blk) for blk in blocks]
    bsp = _spans(counts)
    c = _codec(device)
    L = rans.lib()
    out = np.zeros((max(len(blocks), 1), 2), dtype=np.uint64)
    need = ctypes.c_uint64(0)
    cap = 4 * arena.size + 4096 * len(blocks) + (1 << 16)
    for _ in range(2):
        dst = np.zeros(max(cap, 1), dtype=np.uint8)
        st = L.fqxv_tok_encode_host(c._h, arena.ctypes.data, nsp.ctypes.data, len(names), bsp.ctypes.data,
                                    len(blocks), dst.ctypes.data, dst.size, out.ctypes.data, ctypes.byref(need))
        if st == 17 and need.value > cap:
            cap = need.value
            continue
        _raise(st)
        return [dst[int(o):int(o + n)].tobytes() for o, n in out[:len(blocks)]]
    _raise(17)


def decode_blocks(payloads, device: int = 0, raise_on_error: bool = True):
    """Names of each payload; with raise_on_error False, (names per block,
    statuses) with an empty list for a failed block."""
    payloads = [bytes(p) for p in payloads]
    arena = np.frombuffer(b"".join(payloads) or b"\0", dtype=np.uint8)
    psp = _spans([len(p) for p in payloads])
    n = len(payloads)
    c = _codec(device)
    L = rans.lib()
    blocks = np.zeros((max(n, 1), 2), dtype=np.uint64)
    status = np.zeros(max(n, 1), dtype=np.int32)
    nb, ns = ctypes.c_uint64(0), ctypes.c_uint64(0)
    names_cap, spans_cap = 8 * arena.size + 4096, arena.size + 64
    for _ in range(2):
        h_names = np.zeros(max(names_cap, 1), dtype=np.uint8)
        nsp = np.zeros((max(spans_cap, 1), 2), dtype=np.uint64)
        st = L.fqxv_tok_decode_host(c._h, arena.ctypes.data, psp.ctypes.data, n, h_names.ctypes.data, names_cap,
                                    nsp.ctypes.data, spans_cap, blocks.ctypes.data, status.ctypes.data,
                                    ctypes.byref(nb), ctypes.byref(ns))
        if st == 17 and (nb.value > names_cap or ns.value > spans_cap):
            names_cap, spans_cap = max(nb.value, 1), max(ns.value, 1)
            continue
        break
    if st and st not in TOK_STATUSES and st not in rans.MALFORMED:
        _raise(st)
    out = []
    for b in range(n):
        f, k = int(blocks[b, 0]), int(blocks[b, 1])
        out.append([h_names[int(o):int(o + l)].tobytes() for o, l in nsp[f:f + k]])
    if raise_on_error:
        for s in status[:n]:
            if s:
                _raise(int(s))
        return out
    return out, status[:n].copy()


def encode(names, device: int = 0) -> bytes:
    """lib.rs:482 `encode(names)`."""
    return encode_blocks([list(names)], device)[0]


def decode(src, device: int = 0) -> list[bytes]:
    """lib.rs:543 `decode(src)`."""
    return decode_blocks([src], device)[0]
