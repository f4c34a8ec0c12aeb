"""Harvest the read-name payloads (fqxv-tokenizer v1) stored in the reference's
golden `.fqxv` archives.

Each block of a container stores its read names as one tokenizer payload
(`crates/fqxv-tokenizer/src/lib.rs:482-540`): `[u8 1][varint n_records]`, then
eight `[varint len][rANS stream]` flat / op-run streams and 64 delta-plane
columns. This script walks the archives as bytes (nothing of the reference is
run) and writes every names payload to `fixture_names.bin`, indexed by
`fixture_names.json`. Layouts walked are those of `make_golden.py` (plain
block payloads `[24 digests][u32 n_reads]([u32 len][bytes]) x 3`, names
first; reorder layout names frames).

Run here (where the reference tree is mounted):
    python tests/golden/make_names_golden.py <reference checkout>/crates/fqxv/tests/fixtures

The fixtures directory can also be given as FQXV_FIXTURES in the environment.
"""

from __future__ import annotations

import json
import os
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import FIXTURES, header_len  # noqa: E402


def plain_names(buf: bytes, pos: int) -> list[bytes]:
    out = []
    while True:
        if buf[pos:pos + 4] != b"FQXB":
            raise ValueError("missing block magic at %d" % pos)
        plen = struct.unpack_from("<Q", buf, pos + 4)[0]
        pos += 16
        if plen == 0:
            break
        payload = buf[pos:pos + plen]
        pos += plen
        nlen = struct.unpack_from("<I", payload, 28)[0]
        out.append(payload[32:32 + nlen])
    return out


def reorder_names(buf: bytes, pos: int, flags: int) -> list[bytes]:
    def framed() -> bytes:
        nonlocal pos
        ln = struct.unpack_from("<I", buf, pos)[0]
        data = buf[pos + 8:pos + 8 + ln]
        pos += 8 + ln
        return data

    pos += 8
    framed()
    framed()
    framed()
    if flags & 0x20:
        framed()
    n_blocks = struct.unpack_from("<I", buf, pos)[0]
    pos += 4
    for _ in range(n_blocks):
        framed()
    out = []
    for _ in range(n_blocks):
        out.append(framed())
        framed()
    return out


def main(fixture_dir: str) -> None:
    index = []
    blob = bytearray()
    for name in FIXTURES:
        with open(os.path.join(fixture_dir, name + ".fqxv"), "rb") as f:
            buf = f.read()
        pos, flags = header_len(buf)
        payloads = reorder_names(buf, pos, flags) if flags & 0x08 else plain_names(buf, pos)
        for k, p in enumerate(payloads):
            index.append({"fixture": name, "block": k, "offset": len(blob), "length": len(p)})
            blob += p
    with open(os.path.join(HERE, "fixture_names.bin"), "wb") as f:
        f.write(bytes(blob))
    with open(os.path.join(HERE, "fixture_names.json"), "w") as f:
        json.dump({"source": "crates/fqxv/tests/fixtures/*.fqxv (reference tree)", "payloads": index}, f, indent=1)
    print("%d names payloads, %d bytes" % (len(index), len(blob)))


if __name__ == "__main__":
    fixtures = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FQXV_FIXTURES")
    if not fixtures:
        sys.exit("usage: %s <reference checkout>/crates/fqxv/tests/fixtures (or FQXV_FIXTURES=...)" % sys.argv[0])
    main(fixtures)
