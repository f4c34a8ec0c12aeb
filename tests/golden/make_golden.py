"""Harvest the rANS streams stored inside the reference's golden `.fqxv` archives.

The reference crate has no known-answer vectors at the rANS level; the only
stored rANS bytes in its tree are the name-token streams inside the container
fixtures `crates/fqxv/tests/fixtures/*.fqxv` (written by an earlier release).
This script walks those archives *as bytes* (nothing of the reference is run)
and writes every rANS stream it finds to `fixture_streams.bin`, indexed by
`fixture_streams.json`.

Layouts walked (all little-endian):

* container header: `FQXV`, major, minor, u64 features, k, binning, flags, G,
  platform, u16 ext_len, ext bytes, u32 header CRC
  (`crates/fqxv/src/container/format.rs:195-221`).
* plain layout blocks: `FQXB`, u64 payload length, u32 CRC, payload; a zero
  length ends the block region (`crates/fqxv/src/container/mod.rs:53-63`).
  Payload: 3 x u64 digests, u32 n_reads, then `[u32 len][bytes]` for names,
  sequence, quality (`crates/fqxv/src/container/block.rs:882-923`).
* reorder layout (flags bit 3): u64 n, framed flip / perm / template
  (/ reference when flags bit 5), u32 n_blocks, n framed sequence blocks, then
  n pairs of framed (names, quality); each frame is `[u32 len][u32 crc][bytes]`
  (`crates/fqxv/src/container/reorder.rs:785-802`).
* the names payload is the tokenizer v1 layout: u8 version, varint n_records,
  five flat streams, three op-RLE streams, then 64 delta-plane columns of
  `[varint width]` + width streams; every stream is `[varint len][rANS bytes]`
  (`crates/fqxv-tokenizer/src/lib.rs:98-103, 118-137, 176-200, 482-540`).
* the reorder permutation frame, when non-empty, is one rANS stream
  (`crates/fqxv/src/container/reorder.rs:597-609`).
* a sequence stream with method byte 4 is the long-read tile layout:
  `LRT`, u8 version 1, varint n, varint total_bases, then `put_stream`
  frames `[varint raw_len]([varint enc_len][rANS bytes] when raw_len > 0)`
  for lens, markers, tile_lens, strands, rs, lit_lens, three range-coded
  blobs `[varint count][varint len][bytes]` interleaved after lit_lens and
  runs, then indel_lens, literals, exc_pos, exc_bytes
  (`crates/fqxv-lroverlap/src/tile.rs:714-800`, `codec.rs:293-306`; the
  `put_stream` rule keeps order-1 on a tie).

Run here (where the reference tree is mounted):
    python tests/golden/make_golden.py <reference checkout>/crates/fqxv/tests/fixtures

The fixtures directory can also be given as FQXV_FIXTURES in the environment.
"""

from __future__ import annotations

import json
import os
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = ["plain_se", "paired_labels", "longread", "reorder"]
MAX_COL = 63


def varint(buf: bytes, pos: int) -> tuple[int, int]:
    v = 0
    shift = 0
    while True:
        b = buf[pos]
        pos += 1
        v |= (b & 0x7F) << shift
        if b & 0x80 == 0:
            return v, pos
        shift += 7
        if shift >= 64:
            raise ValueError("over-long varint")


def tokenizer_streams(names: bytes) -> list[tuple[str, bytes]]:
    """Split a tokenizer v1 payload into its rANS streams, labelled by role."""
    out: list[tuple[str, bytes]] = []
    if not names:
        return out
    pos = 0
    if names[pos] != 1:
        raise ValueError("unexpected tokenizer version %d" % names[pos])
    pos += 1
    _, pos = varint(names, pos)  # n_records

    def take(label: str) -> None:
        nonlocal pos
        ln, pos = varint(names, pos)
        out.append((label, names[pos:pos + ln]))
        pos += ln

    for role in ("counts", "str_lens", "str_data", "num_vals", "pads"):
        take(role)
    for role in ("op_run_counts", "op_run_syms", "op_run_lens"):
        take(role)
    for col in range(MAX_COL + 1):
        width, pos = varint(names, pos)
        for plane in range(width):
            take("delta_c%d_p%d" % (col, plane))
    if pos != len(names):
        raise ValueError("tokenizer payload has %d trailing bytes" % (len(names) - pos))
    return out


def tile_streams(seq: bytes) -> list[tuple[str, bytes]]:
    """rANS streams of a long-read tile sequence stream (method byte 4)."""
    out: list[tuple[str, bytes]] = []
    pos = 0
    if seq[pos:pos + 3] != b"LRT" or seq[pos + 3] != 1:
        raise ValueError("not a tile v1 stream")
    pos += 4
    _, pos = varint(seq, pos)  # n
    _, pos = varint(seq, pos)  # total bases

    def put(label: str) -> None:
        nonlocal pos
        raw_len, pos = varint(seq, pos)
        if raw_len == 0:
            return
        ln, pos = varint(seq, pos)
        out.append((label, seq[pos:pos + ln]))
        pos += ln

    def blob() -> None:
        nonlocal pos
        _, pos = varint(seq, pos)
        ln, pos = varint(seq, pos)
        pos += ln

    for role in ("lens", "markers", "tile_lens", "strands", "rs", "lit_lens"):
        put(role)
    blob()  # ops
    put("runs")
    blob()  # subs
    blob()  # ins
    for role in ("indel_lens", "literals", "exc_pos", "exc_bytes"):
        put(role)
    if pos != len(seq):
        raise ValueError("tile stream has %d trailing bytes" % (len(seq) - pos))
    return out


def header_len(buf: bytes) -> tuple[int, int]:
    if buf[:4] != b"FQXV":
        raise ValueError("bad magic")
    flags = buf[16]
    ext_len = struct.unpack_from("<H", buf, 19)[0]
    return 21 + ext_len + 4, flags


def plain_streams(buf: bytes, pos: int) -> list[tuple[str, bytes]]:
    out = []
    blk = 0
    while True:
        if buf[pos:pos + 4] != b"FQXB":
            raise ValueError("missing block magic at %d" % pos)
        plen = struct.unpack_from("<Q", buf, pos + 4)[0]
        pos += 16
        if plen == 0:
            break
        payload = buf[pos:pos + plen]
        pos += plen
        p = 24 + 4
        nlen = struct.unpack_from("<I", payload, p)[0]
        names = payload[p + 4:p + 4 + nlen]
        for role, s in tokenizer_streams(names):
            out.append(("block%d/%s" % (blk, role), s))
        p += 4 + nlen
        slen = struct.unpack_from("<I", payload, p)[0]
        seq = payload[p + 4:p + 4 + slen]
        if seq and seq[0] == 4:
            for role, s in tile_streams(seq[1:]):
                out.append(("block%d/seq_tile/%s" % (blk, role), s))
        blk += 1
    return out


def reorder_streams(buf: bytes, pos: int, flags: int) -> list[tuple[str, bytes]]:
    out = []

    def framed() -> bytes:
        nonlocal pos
        ln = struct.unpack_from("<I", buf, pos)[0]
        data = buf[pos + 8:pos + 8 + ln]
        pos += 8 + ln
        return data

    pos += 8  # n reads
    framed()  # flip bitmap
    perm = framed()
    if perm:
        out.append(("perm", perm))
    framed()  # name template
    if flags & 0x20:
        framed()  # global reference
    n_blocks = struct.unpack_from("<I", buf, pos)[0]
    pos += 4
    for _ in range(n_blocks):
        framed()
    for b in range(n_blocks):
        names = framed()
        framed()  # quality
        for role, s in tokenizer_streams(names):
            out.append(("nqblock%d/%s" % (b, role), s))
    return out


def main(fixture_dir: str) -> None:
    index = []
    blob = bytearray()
    for name in FIXTURES:
        with open(os.path.join(fixture_dir, name + ".fqxv"), "rb") as f:
            buf = f.read()
        pos, flags = header_len(buf)
        streams = reorder_streams(buf, pos, flags) if flags & 0x08 else plain_streams(buf, pos)
        for label, s in streams:
            n = struct.unpack_from("<Q", s, 1)[0] if len(s) >= 9 else None
            index.append({
                "fixture": name,
                "stream": label,
                "offset": len(blob),
                "length": len(s),
                "order": s[0] if s else None,
                "n": n,
            })
            blob += s
    with open(os.path.join(HERE, "fixture_streams.bin"), "wb") as f:
        f.write(bytes(blob))
    with open(os.path.join(HERE, "fixture_streams.json"), "w") as f:
        json.dump({"source": "crates/fqxv/tests/fixtures/*.fqxv (reference tree)",
                   "streams": index}, f, indent=1)
    orders = {}
    for e in index:
        orders[e["order"]] = orders.get(e["order"], 0) + 1
    print("%d streams, %d bytes, orders %s" % (len(index), len(blob), orders))


if __name__ == "__main__":
    fixtures = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FQXV_FIXTURES")
    if not fixtures:
        sys.exit("usage: %s <reference checkout>/crates/fqxv/tests/fixtures (or FQXV_FIXTURES=...)" % sys.argv[0])
    main(fixtures)
