"""Multi-rank host logic on CPU: two gloo ranks shard one batch of blocks,
each codes its share (the oracle stands in for that rank's GPU), and rank 0
reassembles the container order. The result must equal the one-process
encode of the whole batch, and a rank's failure must surface on the host."""

import os
import socket
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, result_path, fail_rank):
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    from fqxv_b200 import shard
    from fqxv_b200 import workloads as W
    from oracle import oracle

    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        data, spans, _ = W.config2(nblocks=40, lo=100, hi=60_000, seed=5)
        parts = shard.partition(spans[:, 1], world)
        mine = parts[rank]
        ok = rank != fail_rank
        streams = []
        if ok:
            for i in mine.tolist():
                o, l = int(spans[i, 0]), int(spans[i, 1])
                blk = data[o:o + l].tobytes()
                e0, e1 = oracle.encode(blk, 0), oracle.encode(blk, 1)
                streams.append(e1 if len(e1) < len(e0) else e0)
        # every rank takes the same collective steps, failed or not
        flags = [None] * world
        dist.all_gather_object(flags, ok)
        gathered = [None] * world
        dist.all_gather_object(gathered, (mine, streams))
        if rank == 0:
            if not all(flags):
                with open(result_path, "w") as f:
                    f.write("rank-failed:%s" % [r for r, x in enumerate(flags) if not x])
                return
            full = shard.assemble(gathered, len(spans))
            blob, out_spans = shard.container_layout(full)
            ref = []
            for o, l in spans.tolist():
                blk = data[o:o + l].tobytes()
                e0, e1 = oracle.encode(blk, 0), oracle.encode(blk, 1)
                ref.append(e1 if len(e1) < len(e0) else e0)
            sizes = [sum(int(spans[i, 1]) for i in p.tolist()) for p in parts]
            with open(result_path, "w") as f:
                f.write("ok" if full == ref and blob == b"".join(ref) else "mismatch")
                f.write(" balance=%.3f" % (max(sizes) / max(1, min(sizes))))
    finally:
        dist.destroy_process_group()


def _run(fail_rank, tmp_path):
    import torch.multiprocessing as mp

    res = tmp_path / "result.txt"
    mp.start_processes(_worker, args=(2, _free_port(), str(res), fail_rank), nprocs=2, join=True,
                       start_method="spawn")
    return res.read_text()


def test_partition_covers_every_block_once():
    from fqxv_b200 import shard

    rng = np.random.default_rng(0)
    lens = rng.integers(1, 1 << 20, 333)
    for world in (1, 2, 3, 8):
        parts = shard.partition(lens, world)
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(len(lens)))
        loads = [int(lens[p].sum()) for p in parts]
        assert max(loads) - min(loads) <= int(lens.max())


def test_two_gloo_ranks_assemble_the_single_process_result(tmp_path):
    out = _run(-1, tmp_path)
    assert out.startswith("ok"), out


def test_failed_rank_is_reported_on_the_host(tmp_path):
    out = _run(1, tmp_path)
    assert out.startswith("rank-failed:[1]"), out
