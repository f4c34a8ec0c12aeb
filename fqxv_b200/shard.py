"""Sharding a batch of independent blocks over several GPUs (one process per
GPU). Blocks are independent, so each rank codes its own subset and nothing
is exchanged on the data path; only the small per-block results (sizes and
streams) travel back to the rank that assembles the container order, the way
the reference's rayon workers each code whole blocks
(crates/fqxv/src/container/compress.rs:868, decompress.rs:46-52).
"""

from __future__ import annotations

import heapq

import numpy as np


def partition(lengths, world: int) -> list[np.ndarray]:
    """Byte-balanced assignment of block indices to `world` ranks: blocks in
    decreasing size go to the least-loaded rank (ties: lowest rank). Each
    rank's list is in ascending block order. Deterministic."""
    lengths = np.asarray(lengths, dtype=np.int64)
    order = sorted(range(len(lengths)), key=lambda i: (-int(lengths[i]), i))
    heap = [(0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(lengths[i]) + 1, r))
    return [np.array(sorted(o), dtype=np.int64) for o in out]


def assemble(per_rank: list[tuple[np.ndarray, list[bytes]]], nblocks: int) -> list[bytes]:
    """Put the per-rank (block indices, streams) back in block order."""
    res: list[bytes | None] = [None] * nblocks
    for idx, streams in per_rank:
        for i, s in zip(idx.tolist(), streams):
            if res[i] is not None:
                raise ValueError("block %d coded twice" % i)
            res[i] = s
    missing = [i for i, s in enumerate(res) if s is None]
    if missing:
        raise ValueError("blocks not coded: %s" % missing[:8])
    return res  # type: ignore[return-value]


def container_layout(streams: list[bytes]) -> tuple[bytes, np.ndarray]:
    """Streams back to back with their (offset, length) spans."""
    lens = np.array([len(s) for s in streams], dtype=np.uint64)
    offs = np.zeros(len(streams), dtype=np.uint64)
    if len(streams):
        offs[1:] = np.cumsum(lens)[:-1]
    return b"".join(streams), np.stack([offs, lens], axis=1)
