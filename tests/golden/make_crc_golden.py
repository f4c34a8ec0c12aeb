"""Harvest every CRC-32C the reference stored in its golden `.fqxv` archives.

The archives `crates/fqxv/tests/fixtures/*.fqxv` (written by an earlier
release of the reference) carry CRC-32C values over known byte ranges. This
script walks them as bytes (nothing of the reference is run) and records, per
CRC, the covered bytes and the stored value:

* header: CRC over the prefix + extension region, stored after it
  (`crates/fqxv/src/container/format.rs:195-221`);
* plain layout block frames `[FQXB][u64 len][u32 crc][payload]`, the CRC over
  the payload (`crates/fqxv/src/container/block.rs:110-142, 1209-1254`);
* reorder layout frames `[u32 len][u32 crc][bytes]` (`format.rs:346-406`,
  `reorder.rs:785-802`);
* plain layout footer (`format.rs:306-343`): each block's three per-stream
  `(offset, len, crc)` triples (`block.rs:961-980`), `whole_file_crc` over
  every byte before it, and `footer_crc` over the footer body.

Output: `fixture_crcs.bin` and `fixture_crcs.json` (per record: fixture,
kind, offset in the archive, length, stored crc, and where its bytes sit in
the .bin). The two small plain archives are kept whole up to the end of the
footer CRC, so every one of their records (whole-file CRC included) has its
bytes; of the two larger archives only records of at most 48 KiB keep their
bytes (the others keep offset, length and CRC, with `bin_offset` null).

Run here (where the reference tree is mounted):
    python tests/golden/make_crc_golden.py <reference checkout>/crates/fqxv/tests/fixtures

The fixtures directory can also be given as FQXV_FIXTURES in the environment.
"""

from __future__ import annotations

import json
import os
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = ["plain_se", "paired_labels", "longread", "reorder"]


def header_records(buf: bytes) -> tuple[list[dict], int, int]:
    if buf[:4] != b"FQXV":
        raise ValueError("bad magic")
    flags = buf[16]
    ext_len = struct.unpack_from("<H", buf, 19)[0]
    covered = 21 + ext_len
    crc = struct.unpack_from("<I", buf, covered)[0]
    return [{"kind": "header", "offset": 0, "length": covered, "crc": crc}], covered + 4, flags


def plain_records(buf: bytes, pos: int) -> list[dict]:
    recs = []
    while True:
        if buf[pos:pos + 4] != b"FQXB":
            raise ValueError("missing block magic at %d" % pos)
        plen = struct.unpack_from("<Q", buf, pos + 4)[0]
        if plen == 0:
            pos += 12
            break
        crc = struct.unpack_from("<I", buf, pos + 12)[0]
        recs.append({"kind": "block_frame", "offset": pos + 16, "length": plen, "crc": crc})
        pos += 16 + plen
    footer_off, magic = struct.unpack_from("<Q4s", buf, len(buf) - 12)
    if magic != b"FQXF" or footer_off != pos:
        return recs
    p = footer_off
    ngroups = struct.unpack_from("<I", buf, p)[0]
    p += 4
    for _ in range(ngroups):
        p += 12
        for _s in range(3):
            s_off, s_len, s_crc = struct.unpack_from("<QII", buf, p)
            p += 16
            recs.append({"kind": "stream_loc", "offset": s_off, "length": s_len, "crc": s_crc})
    p += 8  # total_reads
    whole = struct.unpack_from("<I", buf, p)[0]
    recs.append({"kind": "whole_file", "offset": 0, "length": p, "crc": whole})
    footer_crc = struct.unpack_from("<I", buf, p + 4)[0]
    recs.append({"kind": "footer", "offset": footer_off, "length": p + 4 - footer_off, "crc": footer_crc})
    return recs


def reorder_records(buf: bytes, pos: int, flags: int) -> list[dict]:
    recs = []

    def framed() -> None:
        nonlocal pos
        ln, crc = struct.unpack_from("<II", buf, pos)
        recs.append({"kind": "framed_slice", "offset": pos + 8, "length": ln, "crc": crc})
        pos += 8 + ln

    pos += 8  # n reads
    framed()  # flip bitmap
    framed()  # permutation
    framed()  # name template
    if flags & 0x20:
        framed()  # global reference
    n_blocks = struct.unpack_from("<I", buf, pos)[0]
    pos += 4
    for _ in range(3 * n_blocks):
        framed()
    return recs


WHOLE = ("plain_se", "paired_labels")
MAX_KEPT = 48 << 10


def main(fixture_dir: str) -> None:
    out = []
    blob = bytearray()
    for name in FIXTURES:
        with open(os.path.join(fixture_dir, name + ".fqxv"), "rb") as f:
            buf = f.read()
        recs, pos, flags = header_records(buf)
        recs += reorder_records(buf, pos, flags) if flags & 0x08 else plain_records(buf, pos)
        if name in WHOLE:
            end = max(r["offset"] + r["length"] for r in recs)
            base = len(blob)
            blob += buf[:end]
            for r in recs:
                r["bin_offset"] = base + r["offset"]
        else:
            for r in recs:
                if r["kind"] != "whole_file" and r["length"] <= MAX_KEPT:
                    r["bin_offset"] = len(blob)
                    blob += buf[r["offset"]:r["offset"] + r["length"]]
                else:
                    r["bin_offset"] = None
        for r in recs:
            r["fixture"] = name
            out.append(r)
    with open(os.path.join(HERE, "fixture_crcs.bin"), "wb") as f:
        f.write(bytes(blob))
    with open(os.path.join(HERE, "fixture_crcs.json"), "w") as f:
        json.dump({"source": "crates/fqxv/tests/fixtures/*.fqxv (reference tree)", "records": out}, f, indent=1)
    kinds = {}
    for r in out:
        kinds[r["kind"]] = kinds.get(r["kind"], 0) + 1
    kept = sum(1 for r in out if r["bin_offset"] is not None)
    print("%d records (%d with bytes), %d bytes, %s" % (len(out), kept, len(blob), kinds))


if __name__ == "__main__":
    fixtures = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FQXV_FIXTURES")
    if not fixtures:
        sys.exit("usage: %s <reference checkout>/crates/fqxv/tests/fixtures (or FQXV_FIXTURES=...)" % sys.argv[0])
    main(fixtures)
