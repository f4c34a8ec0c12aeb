#!/usr/bin/env python
"""Throughput benchmark of the B200 rANS Nx16 coder.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload config1]
    python bench.py --impl reference ...      # the CPU arm

A step is one pass of the hot path over one batch: batched encode of every
block of the workload, then batched decode of the streams just written.
`value` is uncompressed GB/s (decimal) of that round trip with the input
resident in HBM, summed over ranks (weak scaling: every rank codes its own
seeded copy of the workload; blocks are independent, there is no collective
on the data path). L2 is flushed (a 256 MiB write) before every timed step.

Workloads (seeded synthetic data of the benchmark shapes):
  config2  4096 mixed blocks 4 KiB - 4 MiB, both orders, keep the smaller
           (tokenizer tie rule)                                    (default)
  config0  1 x 1 MiB binned quality, order-0
  config1  64 x 1 MiB full-range quality, order-1
  config3  config2 (CPU-encoded) + ONT long-read blocks, decode only
  batch0 / batch1 / batch1f   2048 x 512 KiB binned order-0 / binned order-1 /
           full-range order-1: peak batched throughput of one order
  cpu_single (with --impl reference)  the CPU coder on one thread, 8 MiB of
           quality_like data, per path (the reference's own benchmark shape)
  xconfig0 / xconfig2  the extended format (a new format tag, no reference
           counterpart): config 0 as named (4-way, order-0) and config 2 with the
           selection over reference and extended candidates, every stream
           checked against its CPU definition
  names    read-name tokenizer (crates/fqxv-tokenizer): 256 blocks x 4000
           Illumina-style names, encode then decode through the C ABI
  crc      CRC-32C of 4096 payloads 4 KiB - 4 MiB (crates/fqxv/src/crc.rs)
  frame    block frames of the same payloads: write (copy + CRC-32C, terminator)
           then read back with every CRC verified (container/block.rs)

Besides the timed round trip, a run of an encoding workload checks every
stream the GPU wrote against the CPU restatement of the reference encoder
(`byte_identical_blocks`) and decodes the CPU's streams on the GPU; times the
plain one-block-per-launch form of the same batch (`plain_per_block`); and,
on one GPU, runs a short serving pass (`serving`: Poisson arrivals at two
offered loads, p50/p99 latency against plain per-request calls).

The reference arm (`--impl reference`) times the reference's CPU coder -- the
C restatement of fqxv-rans (AVX-512/AVX2 order-0, scalar order-1) -- with all
host threads over the same workload, on rank 0 only.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from fqxv_b200 import workloads as W  # noqa: E402

METRIC = "rANS Nx16 enc/dec GB/s, bit-exact (uncompressed bytes per second, encode + decode round trip)"
L2_FLUSH_BYTES = 256 << 20


def build_workload(name: str, seed: int, blocks: int = 0):
    """-> (data u8, spans (n,2), encode order or None for decode-only, description, extra).

    `blocks` > 0 shrinks configs 1 and 2 to that many blocks (small cases for
    profiler captures); 0 keeps the benchmark shape."""
    if name == "config1":
        nb = blocks or 64
        data, spans = W.config1(nblocks=nb, seed=seed)
        return data, spans, 1, "%d x 1 MiB full-range quality blocks, order-1" % nb, {}
    if name == "config0":
        data, spans = W.config0(seed=seed)
        return data, spans, 0, "1 x 1 MiB binned quality block, order-0", {}
    if name in ("batch0", "batch1", "batch1f"):
        # peak batched throughput of one order: 2048 x 512 KiB (1 GiB)
        kind = "full" if name == "batch1f" else "binned"
        order = 0 if name == "batch0" else 1
        nb = blocks or 2048
        data, spans = W.uniform_batch(kind, nblocks=nb, seed=seed)
        return data, spans, order, "%d x 512 KiB %s quality, order-%d" % (nb, "full-range" if kind == "full" else "binned", order), {}
    workers = min(32, os.cpu_count() or 1)
    if name == "config2":
        nb = blocks or 4096
        data, spans, kinds = W.config2(nblocks=nb, seed=seed, workers=workers)
        return data, spans, 2, "%d mixed blocks 4 KiB-4 MiB, both orders, keep the smaller" % nb, {}
    if name == "config3":
        d2, s2, _ = W.config2(seed=seed, workers=workers)
        d3, s3 = W.config3_ont(seed=seed)
        s3 = s3.copy()
        s3[:, 0] += len(d2)
        data = np.concatenate([d2, d3])
        spans = np.concatenate([s2, s3])
        return data, spans, None, "config2 blocks (CPU-encoded, best order) + ONT quality blocks (order-1), decode", \
            {"n_ont_blocks": int(len(s3))}
    raise SystemExit("unknown workload %s" % name)


FRAME_METRICS = {
    "crc": "CRC-32C GB/s, bit-exact (payload bytes checksummed per second)",
    "frame": "block frames write + verified read GB/s, bit-exact (payload bytes per second)",
}


def frame_workload(seed: int, blocks: int = 0):
    """4096 payloads (log-uniform 4 KiB - 4 MiB, about 2.4 GB) of seeded random
    bytes: the size range of container block payloads, and random bytes stand
    for coded streams (the CRC does the same work on any bytes)."""
    nb = blocks or 4096
    rng = np.random.default_rng(1000 + seed)
    sizes = np.exp(rng.uniform(np.log(4 << 10), np.log(4 << 20), nb)).astype(np.uint64)
    total = int(sizes.sum())
    data = np.frombuffer(rng.bytes(total), dtype=np.uint8)
    offs = np.zeros(nb, dtype=np.uint64)
    offs[1:] = np.cumsum(sizes)[:-1]
    return data, np.stack([offs, sizes], axis=1), "%d payloads 4 KiB-4 MiB, random bytes" % nb


def frame_cpu_step(kind, data, spans, nthreads):
    """The CPU path over the same payloads: CRC-32C of each (crc); or frames
    written (CRC + copy) and read back with each CRC verified (frame)."""
    from oracle import oracle

    if kind == "crc":
        oracle.crc32c_batch(data, spans[:, 0], spans[:, 1], nthreads)
        return
    crcs = oracle.crc32c_batch(data, spans[:, 0], spans[:, 1], nthreads)
    frames = np.empty(int(spans[:, 1].sum()) + 16 * len(spans) + 12, dtype=np.uint8)
    fo = np.zeros(len(spans), dtype=np.uint64)
    fo[1:] = np.cumsum(spans[:, 1] + 16)[:-1]
    for (o, ln), f in zip(spans, fo):
        frames[int(f) + 16:int(f) + 16 + int(ln)] = data[int(o):int(o + ln)]
    got = oracle.crc32c_batch(frames, fo + 16, spans[:, 1], nthreads)
    assert (got == crcs).all()


def run_frames(args, rank: int, world: int, local: int, dist) -> None:
    import torch

    from fqxv_b200.batch import Codec

    kind = args.workload
    data, spans, desc = frame_workload(args.seed + rank, args.blocks)
    n_bytes = int(spans[:, 1].sum())
    codec = Codec(local)
    cs = torch.cuda.ExternalStream(codec.stream_handle)
    d_src = torch.from_numpy(data).to("cuda")
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    need = codec.frame_bound(spans, True)
    d_fr = torch.empty(need, dtype=torch.uint8, device="cuda") if kind == "frame" else None

    def step():
        if kind == "crc":
            return codec.crc32c_batch(d_src, spans)
        _, fo, crcs, total = codec.frame_blocks(d_src, spans, True, d_dst=d_fr)
        pay, rcrcs, st, consumed, term = codec.read_blocks(d_fr, total)
        assert term and consumed == total and not st.any() and (rcrcs == crcs).all()
        return crcs

    from oracle import oracle

    for _ in range(args.warmup):
        crcs = step()
    torch.cuda.synchronize()
    sample = np.linspace(0, len(spans) - 1, 48).astype(int)
    want = [oracle.crc32c(data[int(spans[i, 0]):int(spans[i, 0] + spans[i, 1])]) for i in sample]
    assert [int(crcs[i]) for i in sample] == want, "CRC mismatch against the oracle"
    if kind == "frame":
        fo = np.zeros(len(spans), dtype=np.uint64)
        fo[1:] = np.cumsum(spans[:, 1] + 16)[:-1]
        for i in sample[:8]:
            a, ln = int(fo[i]) + 16, int(spans[i, 1])
            assert torch.equal(d_fr[a:a + ln], d_src[int(spans[i, 0]):int(spans[i, 0]) + ln]), "frame copy mismatch"

    codec.stage_stats(reset=True)
    codec.set_profiling(True)
    sampler = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    total_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(cs)
        step()
        b.record(cs)
        b.synchronize()
        total_ms += a.elapsed_time(b)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    codec.set_profiling(False)
    stages = codec.stage_stats(reset=True)
    t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t[0])
    value = world * n_bytes * args.steps / (total_ms * 1e-3) / 1e9

    pk = peaks()
    timed = {k: v for k, v in stages.items() if v["launches"] > 0}
    dom = max(timed, key=lambda k: timed[k]["ms"])
    launches = timed[dom]["launches"]
    per_launch_ms = timed[dom]["ms"] / launches
    # Algorithmic bytes: the CRC pass reads each payload byte once; the frame
    # copy reads it and writes it once.
    alg_bytes = timed[dom]["bytes"] / launches
    achieved = alg_bytes / (per_launch_ms * 1e-3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            ent = json.load(f).get(kind, {}).get(dom)
        if ent:
            traffic = ent.get("dram_bytes_per_launch")
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 2), "peak": pk["hbm_gbs"],
                "unit": "GB/s", "frac": round(achieved / pk["hbm_gbs"], 5), "traffic": traffic,
                "alg_bytes_per_launch": int(alg_bytes), "launch_ms": round(per_launch_ms, 4),
                "peak_source": pk["source"] + " (MEASURED_PEAKS.json hbm_gbs, copy bandwidth)"}
    gpu_launches = int(sum(v["launches"] for v in stages.values()))

    # end to end through the C ABI with pinned host buffers
    h_src = torch.from_numpy(data).pin_memory().numpy()
    h_fr = torch.empty(need, dtype=torch.uint8).pin_memory().numpy() if kind == "frame" else None

    def e2e_step():
        if kind == "crc":
            return codec.crc32c_batch_host(h_src, spans)
        fo, crcs, total = codec.frame_blocks_host(h_src, spans, h_fr, True)
        pay, rcrcs, st, consumed, term = codec.read_blocks_host(h_fr, total)
        assert term and not st.any() and (rcrcs == crcs).all()
        return crcs

    c = e2e_step()
    assert [int(c[i]) for i in sample] == want, "e2e CRC mismatch"
    e2e_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(cs)
        e2e_step()
        b.record(cs)
        b.synchronize()
        e2e_ms += a.elapsed_time(b)
    t = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_ms = float(t[0])
    e2e = {"value": round(world * n_bytes * args.steps / (e2e_ms * 1e-3) / 1e9, 4), "unit": "GB/s",
           "h2d_bytes_per_step": n_bytes if kind == "crc" else n_bytes + need,
           "d2h_bytes_per_step": 4 * len(spans) if kind == "crc" else need + 4 * len(spans),
           "path": ("fqxv_crc32c_batch_host" if kind == "crc" else
                    "fqxv_frame_blocks_host + fqxv_read_blocks_host") + " (pinned host buffers)"}

    cpu = None
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        nthreads = os.cpu_count() or 1
        sub = spans[:len(spans) // 4]
        sub_bytes = int(sub[:, 1].sum())
        frame_cpu_step(kind, data, sub, nthreads)
        t0 = time.perf_counter()
        reps = 0
        while True:
            frame_cpu_step(kind, data, sub, nthreads)
            reps += 1
            if time.perf_counter() - t0 > 10.0 or reps >= 10:
                break
        dt = time.perf_counter() - t0
        cpu = {"value": round(sub_bytes * reps / dt / 1e9, 4), "unit": "GB/s", "cores": nthreads, "kind": "port",
               "sample": "%d passes over the first quarter of the payloads (%d bytes): the reference's byte-table "
                         "CRC-32C (crc.rs:19-79, restated in C)%s on %d host threads over payloads" %
                         (reps, sub_bytes, "" if kind == "crc" else " + frame copy + verified read", nthreads)}

    if rank == 0:
        line = {
            "metric": FRAME_METRICS[kind], "value": round(value, 4), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": kind, "desc": desc, "blocks": int(len(spans)), "bytes_per_gpu": n_bytes,
                       "l2": "flushed (256 MiB write) before every timed step",
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": gpu_launches,
            "stages": {k: {"launches": v["launches"], "ms": round(v["ms"], 4), "bytes": v["bytes"]}
                       for k, v in stages.items()},
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    codec.close()


def run_frames_reference(args) -> None:
    kind = args.workload
    data, spans, desc = frame_workload(args.seed, args.blocks)
    nthreads = os.cpu_count() or 1
    sub = spans[:len(spans) // 4]
    n_bytes = int(sub[:, 1].sum())
    for _ in range(args.warmup):
        frame_cpu_step(kind, data, sub, nthreads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        frame_cpu_step(kind, data, sub, nthreads)
    dt = time.perf_counter() - t0
    gbs = n_bytes * args.steps / dt / 1e9
    line = {
        "impl": "reference", "metric": FRAME_METRICS[kind], "value": round(gbs, 4), "unit": "GB/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3 / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": kind, "desc": desc, "blocks": int(len(spans)), "bytes": int(spans[:, 1].sum()),
                   "timed_sample_bytes": n_bytes},
        "cpu_baseline": {"value": round(gbs, 4), "unit": "GB/s", "cores": nthreads, "kind": "port",
                         "sample": "the first quarter of the payloads every step: byte-table CRC-32C (crc.rs:19-79, "
                                   "restated in C) on all host threads over payloads"},
        "e2e": {"value": round(gbs, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


NAMES_METRIC = "read-name tokenizer encode + decode GB/s, byte-identical (name bytes per second)"


def names_workload(seed: int, blocks: int = 0):
    """Illumina-style read names `A00123:8:H7KJ2DSXX:<lane>:<tile>:<x>:<y>`, 4000
    per block (the container's block size range), tiles advancing, x / y
    uniform; half the blocks carry the paired-read comment ` 1:N:0:<index>`."""
    nb = blocks or 256
    rng = np.random.default_rng(2000 + seed)
    names, bspans = [], []
    for b in range(nb):
        x = rng.integers(1000, 32000, 4000)
        y = rng.integers(1000, 32000, 4000)
        tile = 1101 + (np.arange(4000) + int(rng.integers(0, 400))) // 400
        suffix = b" 1:N:0:ATCACG" if b % 2 else b""
        first = len(names)
        names += [b"A00123:8:H7KJ2DSXX:%d:%d:%d:%d%s" % (1 + b % 4, tile[i], x[i], y[i], suffix)
                  for i in range(4000)]
        bspans.append((first, 4000))
    lens = np.array([len(n) for n in names], dtype=np.uint64)
    offs = np.zeros(len(names), dtype=np.uint64)
    offs[1:] = np.cumsum(lens)[:-1]
    arena = np.frombuffer(b"".join(names), dtype=np.uint8).copy()
    return (arena, np.ascontiguousarray(np.stack([offs, lens], 1)), np.array(bspans, dtype=np.uint64),
            "%d blocks x 4000 Illumina-style names" % nb)


class NamesCoder:
    """fqxv_tok_encode_host + fqxv_tok_decode_host over one library (the GPU
    library, or the CPU build of the same host code over the oracle coder)."""

    def __init__(self, lib, ctx, arena, nspans, bspans):
        import ctypes

        self.L, self.ctx, self.arena, self.nspans, self.bspans = lib, ctx, arena, nspans, bspans
        vp, sz, u64p = ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint64)
        lib.fqxv_tok_encode_host.argtypes = [vp, vp, vp, sz, vp, sz, vp, ctypes.c_uint64, vp, u64p]
        lib.fqxv_tok_decode_host.argtypes = [vp, vp, vp, sz, vp, ctypes.c_uint64, vp, ctypes.c_uint64, vp, vp,
                                             u64p, u64p]
        self.nb = len(bspans)
        self.pay = np.zeros(arena.size + 8192 * self.nb, dtype=np.uint8)
        self.pspans = np.zeros((self.nb, 2), dtype=np.uint64)
        self.names = np.zeros(arena.size, dtype=np.uint8)
        self.out_nspans = np.zeros((len(nspans), 2), dtype=np.uint64)
        self.out_b = np.zeros((self.nb, 2), dtype=np.uint64)
        self.status = np.zeros(self.nb, dtype=np.int32)
        self.c = ctypes

    def encode(self):
        need = self.c.c_uint64(0)
        st = self.L.fqxv_tok_encode_host(self.ctx, self.arena.ctypes.data, self.nspans.ctypes.data, len(self.nspans),
                                         self.bspans.ctypes.data, self.nb, self.pay.ctypes.data, self.pay.size,
                                         self.pspans.ctypes.data, self.c.byref(need))
        assert st == 0, st
        return int(need.value)

    def decode(self):
        a, b = self.c.c_uint64(0), self.c.c_uint64(0)
        st = self.L.fqxv_tok_decode_host(self.ctx, self.pay.ctypes.data, self.pspans.ctypes.data, self.nb,
                                         self.names.ctypes.data, self.names.size, self.out_nspans.ctypes.data,
                                         len(self.out_nspans), self.out_b.ctypes.data, self.status.ctypes.data,
                                         self.c.byref(a), self.c.byref(b))
        assert st == 0 and not self.status.any(), st

    def check(self):
        assert np.array_equal(self.names, self.arena) and np.array_equal(self.out_nspans, self.nspans)


def names_cpu_rate(arena, nspans, bspans, k: int):
    """The CPU build of the tokenizer host code over the oracle coder, all host
    threads, on the first k blocks: (GB/s, reps, bytes, threads)."""
    import ctypes

    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    L = ctypes.CDLL(os.path.join(ROOT, "oracle", "_build", "libcallers_cpu.so"))
    sub_b = bspans[:k]
    n_names = int(sub_b[-1, 0] + sub_b[-1, 1])
    sub_n = nspans[:n_names]
    nbytes = int(sub_n[-1, 0] + sub_n[-1, 1])
    coder = NamesCoder(L, ctypes.c_void_p(1), arena[:nbytes].copy(), sub_n.copy(), sub_b.copy())
    coder.encode()
    coder.decode()
    coder.check()
    t0 = time.perf_counter()
    reps = 0
    while time.perf_counter() - t0 < 10.0 and reps < 20:
        coder.encode()
        coder.decode()
        reps += 1
    dt = time.perf_counter() - t0
    return nbytes * reps / dt / 1e9, reps, nbytes, os.cpu_count() or 1


def run_names(args, rank: int, world: int, local: int, dist) -> None:
    import torch

    from fqxv_b200 import frame, rans

    arena, nspans, bspans, desc = names_workload(args.seed + rank, args.blocks)
    n_bytes = int(arena.size)
    codec = frame.codec(local)
    coder = NamesCoder(rans.lib(), codec._h, arena, nspans, bspans)
    for _ in range(args.warmup):
        payload_bytes = coder.encode()
        coder.decode()
    coder.check()
    codec.stage_stats(reset=True)
    codec.set_profiling(True)
    sampler = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    enc_s = dec_s = 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        coder.encode()
        t1 = time.perf_counter()
        coder.decode()
        t2 = time.perf_counter()
        enc_s += t1 - t0
        dec_s += t2 - t1
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    codec.set_profiling(False)
    stages = codec.stage_stats(reset=True)
    total_s = enc_s + dec_s
    t = torch.tensor([total_s, enc_s], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_s, enc_s = float(t[0]), float(t[1])
    value = world * n_bytes * args.steps / total_s / 1e9
    pk = peaks()
    timed = {k: v for k, v in stages.items() if v["launches"] > 0}
    dom = max(timed, key=lambda k: timed[k]["ms"])
    per_launch_ms = timed[dom]["ms"] / timed[dom]["launches"]
    alg_bytes = timed[dom]["bytes"] / timed[dom]["launches"]
    achieved = alg_bytes / (per_launch_ms * 1e-3) / 1e9
    gpu_ms = sum(v["ms"] for v in timed.values()) / args.steps
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 2), "peak": pk["hbm_gbs"],
                "unit": "GB/s", "frac": round(achieved / pk["hbm_gbs"], 6), "traffic": None,
                "alg_bytes_per_launch": int(alg_bytes), "launch_ms": round(per_launch_ms, 4),
                "peak_source": pk["source"] + " (MEASURED_PEAKS.json hbm_gbs, copy bandwidth)"}
    cpu = None
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        rate, reps, nb_s, thr = names_cpu_rate(arena, nspans, bspans, min(32, len(bspans)))
        cpu = {"value": round(rate, 4), "unit": "GB/s", "cores": thr, "kind": "port",
               "sample": "%d encode + decode passes over the first 32 blocks (%d name bytes): the tokenizer host "
                         "code over the C restatement of the fqxv-rans CPU coder (both orders, keep the smaller), "
                         "streams spread over %d host threads" % (reps, nb_s, thr)}
    if rank == 0:
        line = {
            "metric": NAMES_METRIC, "value": round(value, 4), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_s * 1e3 / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": "names", "desc": desc, "blocks": int(len(bspans)), "names": int(len(nspans)),
                       "bytes_per_gpu": n_bytes, "payload_bytes_per_gpu": payload_bytes,
                       "timing": "host clock around the synchronous C-ABI calls (host buffers in and out), so "
                                 "value is end to end; GPU kernel time per step in gpu_ms_per_step",
                       "l2": "inputs come from host memory every step",
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "encode_gbs": round(world * n_bytes * args.steps / enc_s / 1e9, 4),
            "decode_gbs": round(world * n_bytes * args.steps / (total_s - enc_s) / 1e9, 4),
            "gpu_ms_per_step": round(gpu_ms, 3),
            "roofline": roofline, "cpu_baseline": cpu,
            "e2e": {"value": round(value, 4), "unit": "GB/s", "h2d_bytes_per_step": n_bytes + payload_bytes,
                    "d2h_bytes_per_step": n_bytes + payload_bytes,
                    "path": "fqxv_tok_encode_host + fqxv_tok_decode_host (host buffers)"},
            "gpu_launches": int(sum(v["launches"] for v in stages.values())),
            "stages": {k: {"launches": v["launches"], "ms": round(v["ms"], 4), "bytes": v["bytes"]}
                       for k, v in stages.items() if v["launches"]},
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)


def run_names_reference(args) -> None:
    arena, nspans, bspans, desc = names_workload(args.seed, args.blocks)
    rate, reps, nb_s, thr = names_cpu_rate(arena, nspans, bspans, min(32, len(bspans)))
    line = {"impl": "reference", "metric": NAMES_METRIC, "value": round(rate, 4), "unit": "GB/s",
            "n_gpus": args.gpus, "steps": reps, "warmup": 1, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": "names", "desc": desc, "timed_sample_bytes": nb_s},
            "cpu_baseline": {"value": round(rate, 4), "unit": "GB/s", "cores": thr, "kind": "port",
                             "sample": "the first 32 blocks: tokenizer host code over the C restatement of the "
                                       "fqxv-rans CPU coder on all host threads"},
            "e2e": {"value": round(rate, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


X_METRIC = "extended format (4-way cores, STRIPE/RLE/PACK/CAT) enc/dec GB/s, identical to its CPU definition"


def run_xformat(args, rank: int, world: int, local: int, dist) -> None:
    """xconfig0: config 0 as named -- one 1 MiB block of binned quality,
    order-0, 4-way interleave (flags 0x02). xconfig2: config 2's 4096 mixed
    blocks, the selection over reference and extended candidates (0x40).
    A step is the GPU encode of every block then the decode of its streams;
    every stream is checked against the CPU definition (oracle/rans_x.c,
    parity unpinned against the reference, which has no such format)."""
    import torch

    from fqxv_b200.batch import Codec
    from oracle import oracle

    if args.workload == "xconfig0":
        data, spans = W.config0(seed=args.seed + rank)
        flags, desc = 0x02, "1 x 1 MiB binned quality, order-0, 4-way interleave"
    else:
        data, spans, _ = W.config2(nblocks=args.blocks or 4096, seed=args.seed + rank,
                                   workers=min(32, os.cpu_count() or 1))
        flags, desc = 0x40, "%d mixed blocks 4 KiB-4 MiB, smallest of reference and extended candidates" % len(spans)
    n_bytes = int(spans[:, 1].sum())
    codec = Codec(local)
    cs = torch.cuda.ExternalStream(codec.stream_handle)
    d_src = torch.from_numpy(data).to("cuda")
    d_dec = torch.empty(max(n_bytes, 1), dtype=torch.uint8, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    def step():
        d_enc, es, ch = codec.x_encode_batch(d_src, spans, flags)
        _, lens, st = codec.x_decode_batch(d_enc, es, spans, d_dst=d_dec)
        return d_enc, es, ch, st

    for _ in range(args.warmup):
        d_enc, es, ch, st = step()
    torch.cuda.synchronize()
    assert (st == 0).all() and torch.equal(d_dec[:n_bytes], d_src[:n_bytes]), "round trip mismatch"
    identity = None
    if rank == 0 and not args.no_identity:
        ref, roff, rlen, rch = oracle.x_encode_batch(data, spans[:, 0], spans[:, 1], flags)
        got = d_enc[:int(es[-1, 0] + es[-1, 1])].cpu().numpy()
        same = sum(1 for i in range(len(spans)) if int(es[i, 1]) == int(rlen[i]) and np.array_equal(
            got[int(es[i, 0]):int(es[i, 0] + es[i, 1])], ref[int(roff[i]):int(roff[i] + rlen[i])]))
        kinds = {int(k): int((rch == k).sum()) for k in np.unique(rch)}
        identity = {"blocks": "%d/%d" % (same, len(spans)), "choices_equal": bool((ch == rch).all()),
                    "choice_counts": kinds}
    codec.stage_stats(reset=True)
    codec.set_profiling(True)
    sampler = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    total_ms = 0.0
    comp = 0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(cs)
        d_enc, es, ch, st = step()
        b.record(cs)
        b.synchronize()
        total_ms += a.elapsed_time(b)
        comp = int(es[:, 1].sum())
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    codec.set_profiling(False)
    stages = codec.stage_stats(reset=True)
    t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t[0])
    value = world * n_bytes * args.steps / (total_ms * 1e-3) / 1e9
    cpu = None
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        nthreads = os.cpu_count() or 1
        t0 = time.perf_counter()
        reps = 0
        while time.perf_counter() - t0 < 5.0 and reps < 5:
            oracle.x_encode_batch(data, spans[:, 0], spans[:, 1], flags, nthreads)
            reps += 1
        dt = time.perf_counter() - t0
        cpu = {"value": round(n_bytes * reps / dt / 1e9, 4), "unit": "GB/s", "cores": nthreads, "kind": "port",
               "sample": "%d encode passes of the whole workload by the CPU definition (oracle/rans_x.c) on %d "
                         "host threads" % (reps, nthreads)}
    if rank == 0:
        line = {
            "metric": X_METRIC, "value": round(value, 4), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": args.workload, "desc": desc, "blocks": int(len(spans)), "bytes_per_gpu": n_bytes,
                       "compressed_bytes_per_gpu": comp, "flags": flags,
                       "l2": "flushed (256 MiB write) before every timed step",
                       "parity": "against the CPU definition; unpinned against the reference (no such format)"},
            "identity": identity, "cpu_baseline": cpu,
            "gpu_launches": int(sum(v["launches"] for v in stages.values())),
            "stages": {k: {"launches": v["launches"], "ms": round(v["ms"], 4), "wall_ms": round(v["wall_ms"], 4)}
                       for k, v in stages.items() if v["launches"]},
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    codec.close()


def peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled every few
    milliseconds through NVML while the timed region runs (reads only; no
    setting of the GPU is changed). Falls back to `nvidia-smi -lms 100`."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, index: int):
        self.index = index
        self.sm: list[float] = []
        self.smax = None
        self.reasons: set[str] = set()
        self.stop_flag = threading.Event()
        self.t = None
        self.proc = None
        self.lines: list[str] = []
        self.nvml = None

    def _nvml_handle(self):
        import pynvml

        pynvml.nvmlInit()
        try:
            import torch

            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            self.nvml = (nv, h)
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _poll(self):
        nv, h = self.nvml
        while not self.stop_flag.is_set():
            try:
                self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                for name, const in self.REASONS:
                    if r & getattr(nv, const):
                        self.reasons.add(name)
            except Exception:
                return
            time.sleep(0.002)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        self.stop_flag.set()
        if self.nvml:
            self.t.join(timeout=2)
            src = "nvml, 2 ms"
        elif self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)
            smax = []
            for ln in self.lines:
                parts = [x.strip() for x in ln.split(",")]
                if len(parts) < 6:
                    continue
                try:
                    self.sm.append(float(parts[0]))
                    smax.append(float(parts[1]))
                except ValueError:
                    continue
                for (nm, _), v in zip(self.REASONS, parts[2:6]):
                    if v.lower() == "active":
                        self.reasons.add(nm)
            self.smax = max(smax) if smax else None
            src = "nvidia-smi, 100 ms"
        else:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no clock source"], "samples": 0}
        if not self.sm:
            return {"sm_mhz": None, "sm_max_mhz": self.smax, "reasons": ["no samples"], "samples": 0}
        return {"sm_mhz": float(np.median(self.sm)), "sm_max_mhz": self.smax, "reasons": sorted(self.reasons),
                "samples": len(self.sm), "source": src}


def oracle_roundtrip(data, spans, order, nthreads=0):
    """One CPU pass: encode every block then decode it (the reference's
    rayon-over-blocks shape on all host threads). Returns (enc arena, offs, lens)."""
    from oracle import oracle

    enc, eoff, elen = oracle.encode_batch(data, spans[:, 0], spans[:, 1], order, nthreads)
    dec, _, dlen = oracle.decode_batch(enc, eoff, elen, spans[:, 1], nthreads)
    return enc, eoff, elen


def cpu_encoded(data, spans, seed_tag):
    """CPU-encoded streams for the decode-only workload (reference encoder,
    best order with the tokenizer's tie rule)."""
    from oracle import oracle

    enc, eoff, elen = oracle.encode_batch(data, spans[:, 0], spans[:, 1], 2)
    # compact
    parts = [enc[int(o):int(o + l)] for o, l in zip(eoff, elen)]
    arena = np.concatenate(parts) if parts else np.zeros(0, np.uint8)
    offs = np.zeros(len(parts), np.uint64)
    if len(parts):
        offs[1:] = np.cumsum(elen)[:-1]
    return arena, np.stack([offs, elen.astype(np.uint64)], 1)


def run_cpu_single(args) -> None:
    """One thread, 8 MiB of `quality_like` data (the shape of the
    reference's own criterion benchmarks, benches/rans.rs:11-25): MiB/s of
    the CPU restatement per path, to set beside the reference's published
    single-thread figures (lib.rs:15-16, 106-108, 176-178)."""
    from oracle import oracle

    data = W.quality_like(8 << 20).tobytes()
    n = len(data)
    paths = ["scalar"] + (["avx2"] if oracle.simd_level() >= 1 else []) + (["avx512"] if oracle.simd_level() >= 2 else [])
    rows = {}

    def rate(fn):
        fn()
        t0 = time.perf_counter()
        reps = 0
        while time.perf_counter() - t0 < 1.0 or reps < 3:
            fn()
            reps += 1
        return round(n * reps / (time.perf_counter() - t0) / (1 << 20), 1)

    for path in paths:
        enc = oracle.encode(data, 0, path=path)
        rows["order0_encode_" + path] = rate(lambda: oracle.encode(data, 0, path=path))
        rows["order0_decode_" + path] = rate(lambda: oracle.decode(enc, path=path))
    enc1 = oracle.encode(data, 1)
    rows["order1_encode_scalar"] = rate(lambda: oracle.encode(data, 1))
    rows["order1_decode_scalar"] = rate(lambda: oracle.decode(enc1))
    line = {"impl": "reference", "metric": "single-thread CPU MiB/s (8 MiB quality_like)", "unit": "MiB/s",
            "config": {"workload": "cpu_single", "bytes": n, "threads": 1}, "rates": rows,
            "published_cascade_lake": {"order0_decode_scalar": 163, "order0_decode_avx2": 315,
                                       "order0_decode_avx512": 817, "order0_encode_scalar": 163,
                                       "order0_encode_avx512": 233}}
    print(json.dumps(line), flush=True)


def run_reference(args, rank: int) -> None:
    if rank != 0:
        return
    if args.workload == "cpu_single":
        run_cpu_single(args)
        return
    if args.workload in FRAME_METRICS:
        run_frames_reference(args)
        return
    if args.workload == "names":
        run_names_reference(args)
        return
    if args.workload.startswith("x"):
        print(json.dumps({"impl": "reference", "unavailable": "fqxv-rans writes only its 32-way untagged format; the "
                          "extended format has no reference implementation (crates/fqxv-rans/src/model.rs:19, "
                          "scalar.rs:8-20)"}), flush=True)
        return
    data, spans, order, desc, extra = build_workload(args.workload, args.seed, args.blocks)
    nthreads = os.cpu_count() or 1
    n_bytes = int(spans[:, 1].sum())
    from oracle import oracle

    if order is None:
        arena, cspans = cpu_encoded(data, spans, args.seed)

        def step():
            oracle.decode_batch(arena, cspans[:, 0], cspans[:, 1], spans[:, 1], nthreads)
    else:
        def step():
            oracle_roundtrip(data, spans, order, nthreads)
    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    gbs = n_bytes * args.steps / dt / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(gbs, 4), "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3 / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": dict({"workload": args.workload, "desc": desc, "blocks": int(len(spans)), "bytes": n_bytes}, **extra),
        "cpu_baseline": {"value": round(gbs, 4), "unit": "GB/s", "cores": nthreads, "kind": "port",
                         "sample": "the whole workload every step (C restatement of fqxv-rans: AVX-512/AVX2 "
                                   "order-0, scalar order-1), all host threads over blocks"},
        "e2e": {"value": round(gbs, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def serving_levels(seed: int, nreq: int, loads, workers: int) -> dict:
    """config4's serving loop: requests arrive as a Poisson process at offered
    loads (fractions of the measured batched capacity); 70% decompress / 30%
    compress; sizes log-uniform 16 KiB - 64 MiB; stream types of configs 2
    and 3. The server admits by device memory under a 40 GB cap and batches
    continuously; the same schedule also runs through plain per-request
    calls. Returns the capacity and, per load, p50/p99 of both forms and
    whether every result is byte-identical to the expected stream."""
    import queue as _queue

    import torch

    from fqxv_b200 import rans
    from fqxv_b200.serve import Server
    from oracle import oracle

    rng = np.random.default_rng(seed)
    kinds = ["binned", "full", "acgt", "names", "ont"]
    reqs = []
    for i in range(nreq):
        size = int(np.exp(rng.uniform(np.log(16 << 10), np.log(64 << 20))))
        kind = kinds[int(rng.integers(0, len(kinds)))]
        if kind == "ont":
            data = W.ont_reads(max(1, size // 8000 + 1), seed + i)[:size]
        else:
            data = W.GENERATORS[kind](size, seed + i)
        raw = data.tobytes()
        e0, e1 = oracle.encode(raw, 0), oracle.encode(raw, 1)
        best = e1 if len(e1) < len(e0) else e0
        if rng.random() < 0.7:
            reqs.append(("dec", best, len(raw), raw))
        else:
            reqs.append(("enc", raw, len(raw), best))
    total = sum(r[2] for r in reqs)
    torch.cuda.init()

    # One long-lived server (created and warmed once, as in deployment).
    srv = Server(device=0, workers=workers, hbm_cap=40 << 30)

    def run_server(arrivals):
        lat = [0.0] * nreq
        b0 = srv.stats()["batches"]
        ids = [None] * nreq
        t0 = time.perf_counter()
        for i, (k, d, n, _) in enumerate(reqs):
            wait = arrivals[i] - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
            ids[i] = srv.submit_decode(d) if k == "dec" else srv.submit_encode(d, rans.Order.BestTie0)
        outs = []
        for i in range(nreq):
            outs.append(srv.result(ids[i]))
            lat[i] = srv.last_latency_us / 1e3
        wall = time.perf_counter() - t0
        st = srv.stats()
        st["batches"] -= b0
        return outs, lat, wall, st

    def run_plain(arrivals):
        # one request at a time through the single-call C ABI, in arrival order
        lat = [0.0] * nreq
        q = _queue.Queue()
        done = [None] * nreq
        outs = [None] * nreq

        def worker():
            while True:
                item = q.get()
                if item is None:
                    return
                i, t_arr = item
                k, d, n, _ = reqs[i]
                outs[i] = rans.decode(d) if k == "dec" else rans.encode(d, rans.Order.BestTie0)
                done[i] = time.perf_counter()
        th = threading.Thread(target=worker)
        th.start()
        t0 = time.perf_counter()
        arr_abs = [0.0] * nreq
        for i in range(nreq):
            wait = arrivals[i] - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
            arr_abs[i] = time.perf_counter()
            q.put((i, arr_abs[i]))
        q.put(None)
        th.join()
        wall = time.perf_counter() - t0
        for i in range(nreq):
            lat[i] = (done[i] - arr_abs[i]) * 1e3
        return outs, lat, wall

    # expected result of each request: the original bytes (decompress) or
    # the reference encoder's best-order stream (compress)
    expect = [r[3] for r in reqs]
    # warm-up pass, then capacity: everything submitted at once
    run_server([0.0] * nreq)
    outs, lat, wall, st = run_server([0.0] * nreq)
    cap_ok = all(o == e for o, e in zip(outs, expect))
    cap_gbs = total / wall / 1e9
    levels = []
    for load in loads:
        lam = load * cap_gbs * 1e9 / (total / nreq)  # requests per second
        arrivals = list(np.cumsum(np.random.default_rng(seed + int(load * 100)).exponential(1.0 / lam, nreq)))
        outs, lat, wall, st = run_server(arrivals)
        same = all(o == e for o, e in zip(outs, expect))
        outs_p, lat_p, wall_p = run_plain(arrivals)
        same_p = all(o == e for o, e in zip(outs_p, expect))
        levels.append({
            "offered_load": load, "offered_gbs": round(load * cap_gbs, 3),
            "served": {"gbs": round(total / wall / 1e9, 3), "p50_ms": round(float(np.percentile(lat, 50)), 2),
                       "p99_ms": round(float(np.percentile(lat, 99)), 2), "batches": st["batches"],
                       "byte_identical": bool(same)},
            "plain_per_request": {"gbs": round(total / wall_p / 1e9, 3),
                                  "p50_ms": round(float(np.percentile(lat_p, 50)), 2),
                                  "p99_ms": round(float(np.percentile(lat_p, 99)), 2),
                                  "byte_identical": bool(same_p)},
        })
    srv.close()
    return {"requests": nreq, "bytes": total, "capacity_gbs": round(cap_gbs, 3), "capacity_byte_identical": cap_ok,
            "levels": levels}


def run_serving(args, rank: int) -> None:
    """config4 on its own line: every offered load of --loads."""
    if rank != 0:
        return
    res = serving_levels(args.seed, args.requests, args.loads, args.workers)
    levels = res["levels"]
    line = {
        "metric": "rANS Nx16 serving: p50/p99 latency vs offered load (GB/s of uncompressed bytes)",
        "value": levels[-1]["served"]["gbs"], "unit": "GB/s", "n_gpus": 1, "steps": len(args.loads),
        "warmup": 1, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8", "data": "synthetic",
        "config": {"workload": "config4", "requests": res["requests"], "bytes": res["bytes"],
                   "decompress_fraction": 0.7, "sizes": "log-uniform 16 KiB - 64 MiB", "hbm_cap_bytes": 40 << 30,
                   "workers": args.workers},
        "capacity_gbs": res["capacity_gbs"], "levels": levels,
    }
    print(json.dumps(line), flush=True)


def check_identity(codec, data, spans, order, d_enc, enc_spans, decode_only) -> dict:
    """Every stream the GPU wrote against the CPU restatement of the
    reference encoder (same order mode, same tie rule), block by block; and
    the CPU's streams decoded on the GPU against the input. Decode-only
    workloads check the GPU decode of the CPU's streams only."""
    import torch

    from oracle import oracle

    nthreads = os.cpu_count() or 1
    n_bytes = int(spans[:, 1].sum())
    out = {}
    if not decode_only:
        ref, roff, rlen = oracle.encode_batch(data, spans[:, 0], spans[:, 1], order, nthreads)
        total = int(enc_spans[-1, 0] + enc_spans[-1, 1])
        got = d_enc[:total].cpu().numpy()
        same = 0
        for i in range(len(spans)):
            o, ln = int(enc_spans[i, 0]), int(enc_spans[i, 1])
            if ln == int(rlen[i]) and np.array_equal(got[o:o + ln], ref[int(roff[i]):int(roff[i] + rlen[i])]):
                same += 1
        out["blocks"] = "%d/%d" % (same, len(spans))
        out["encoder"] = "oracle.encode_batch mode %d (C restatement of fqxv-rans scalar.rs/model.rs)" % order
        arena, cspans = ref, np.stack([roff, rlen], 1)
    else:
        arena, cspans = cpu_encoded(data, spans, 0)
    d_ref = torch.from_numpy(np.ascontiguousarray(arena)).to("cuda")
    d_dec, lens, st = codec.decode_batch(d_ref, cspans, spans)
    torch.cuda.synchronize()
    ok = bool((st == 0).all()) and np.array_equal(d_dec[:n_bytes].cpu().numpy(), data[:n_bytes])
    out["cpu_streams_gpu_decoded"] = ok
    if decode_only:
        out["blocks"] = "%d/%d" % (int((st == 0).sum()) if ok else 0, len(spans))
    assert ok, "GPU decode of the CPU encoder's streams differs from the input"
    del d_ref, d_dec
    return out


def stage_roofline(stages: dict, steps: int, workload: str) -> dict:
    """The dominant stage against the HBM roofline. A stage can be several
    launches that run side by side on separate CUDA streams (the decode
    groups), so its time is its wall time on the device per step (first
    launch start to last launch end), and its algorithmic bytes are those of
    all its launches in the step: decode moves compressed + n bytes of the
    streams it decodes, encode n + the words written, pack the words read +
    the stream written; tables are on chip and excluded."""
    pk = peaks()
    timed = {k: v for k, v in stages.items() if v["launches"] > 0}
    dom = max(timed, key=lambda k: timed[k]["wall_ms"])
    wall_ms = timed[dom]["wall_ms"] / steps
    alg_bytes = timed[dom]["bytes"] / steps
    achieved = alg_bytes / (wall_ms * 1e-3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            tr = json.load(f)
        ent = tr.get(workload, {}).get(dom)
        if ent:
            traffic = ent.get("dram_bytes_per_step")
    return {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 2), "peak": pk["hbm_gbs"],
            "unit": "GB/s", "frac": round(achieved / pk["hbm_gbs"], 6), "traffic": traffic,
            "alg_bytes_per_step": int(alg_bytes), "wall_ms_per_step": round(wall_ms, 4),
            "launches_per_step": timed[dom]["launches"] / steps,
            "peak_source": pk["source"] + " (MEASURED_PEAKS.json hbm_gbs, copy bandwidth)"
            if pk["source"] == "measured" else "fallback 6650 GB/s (MEASURED_PEAKS.json absent)"}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="config2",
                    choices=["config1", "config0", "config2", "config3", "config4", "batch0", "batch1", "batch1f",
                             "cpu_single", "crc", "frame", "names", "xconfig0", "xconfig2"])
    ap.add_argument("--requests", type=int, default=48, help="config4: requests per load level")
    ap.add_argument("--workers", type=int, default=8, help="config4: server workers (streams)")
    ap.add_argument("--loads", type=float, nargs="+", default=[0.25, 0.5, 0.75, 1.0])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--blocks", type=int, default=0,
                    help="configs 1/2 and batch*: number of blocks (0 = the benchmark shape; smaller for profiler captures)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-identity", action="store_true",
                    help="skip the check of every GPU stream against the CPU encoder")
    ap.add_argument("--serving-requests", type=int, default=24,
                    help="requests of the serving pass in the default line (0: no serving pass)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.workload == "config4":
        run_serving(args, rank)
        return

    import torch

    from fqxv_b200.batch import Codec

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    if args.workload in FRAME_METRICS or args.workload in ("names", "xconfig0", "xconfig2"):
        fn = run_names if args.workload == "names" else run_xformat if args.workload.startswith("x") else run_frames
        fn(args, rank, world, local, dist)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    data, spans, order, desc, extra = build_workload(args.workload, args.seed + rank, args.blocks)
    n_bytes = int(spans[:, 1].sum())
    codec = Codec(local)
    cs = torch.cuda.ExternalStream(codec.stream_handle)
    d_src = torch.from_numpy(data).to("cuda")
    d_dec = torch.empty(max(n_bytes, 1), dtype=torch.uint8, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    decode_only = order is None
    if decode_only:
        arena, cspans = cpu_encoded(data, spans, args.seed)
        d_enc = torch.from_numpy(arena).to("cuda")
        enc_spans = cspans
        comp_bytes = int(cspans[:, 1].sum())
    else:
        d_enc = torch.empty(max(codec.encode_bound(spans, order), 1), dtype=torch.uint8, device="cuda")
        enc_spans = None
        comp_bytes = 0

    def step(persistent=True):
        nonlocal enc_spans, comp_bytes
        if not decode_only:
            _, enc_spans, _ = codec.encode_batch(d_src, spans, order, d_dst=d_enc, persistent=persistent)
            comp_bytes = int(enc_spans[:, 1].sum())
        _, lens, st = codec.decode_batch(d_enc, enc_spans, spans, d_dst=d_dec, persistent=persistent)
        return st

    for _ in range(args.warmup):
        st = step()
    torch.cuda.synchronize()
    assert (st == 0).all() and torch.equal(d_dec[:n_bytes], d_src[:n_bytes]), "round trip mismatch"

    # ---- byte identity against the CPU encoder (outside the timed region) -----
    identity = None
    if not args.no_identity and rank == 0:
        identity = check_identity(codec, data, spans, order, d_enc, enc_spans, decode_only)

    # ---- timed region ---------------------------------------------------
    codec.stage_stats(reset=True)
    codec.set_profiling(True)
    sampler = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    total_ms = 0.0
    enc_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(cs)
        if not decode_only:
            _, enc_spans, _ = codec.encode_batch(d_src, spans, order, d_dst=d_enc)
        e1.record(cs)
        codec.decode_batch(d_enc, enc_spans, spans, d_dst=d_dec)
        e2.record(cs)
        e2.synchronize()
        total_ms += e0.elapsed_time(e2)
        enc_ms += e0.elapsed_time(e1)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    codec.set_profiling(False)
    stages = codec.stage_stats(reset=True)
    if not decode_only:
        comp_bytes = int(enc_spans[:, 1].sum())

    t = torch.tensor([total_ms, enc_ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms, enc_ms = float(t[0]), float(t[1])
    dec_ms = total_ms - enc_ms
    value = world * n_bytes * args.steps / (total_ms * 1e-3) / 1e9

    # ---- the dominant kernel against the HBM roofline -------------------------
    roofline = stage_roofline(stages, args.steps, args.workload)
    gpu_launches = int(sum(v["launches"] for v in stages.values()))

    # ---- plain one-block-per-launch form (same bytes) -------------------------
    plain = None
    if not args.no_plain and rank == 0:
        flush.zero_()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(cs)
        st = step(persistent=False)
        b.record(cs)
        b.synchronize()
        ok = bool((st == 0).all()) and torch.equal(d_dec[:n_bytes], d_src[:n_bytes])
        pg = n_bytes / (a.elapsed_time(b) * 1e-3) / 1e9
        own = n_bytes * args.steps / (total_ms * 1e-3) / 1e9
        plain = {"gbs": round(pg, 4), "round_trip_ok": ok, "batched_over_plain": round(own / pg, 2),
                 "form": "one launch per block and stage, same kernels, same bytes"}

    # ---- end to end through the C ABI with pinned host buffers ---------------
    h_src = torch.from_numpy(data).pin_memory().numpy()
    h_dec = torch.empty(max(n_bytes, 1), dtype=torch.uint8).pin_memory().numpy()
    if decode_only:
        h_enc = torch.from_numpy(arena).pin_memory().numpy()
    else:
        h_enc = torch.empty(max(codec.encode_bound(spans, order), 1), dtype=torch.uint8).pin_memory().numpy()

    def e2e_step():
        if decode_only:
            es = enc_spans
        else:
            es, _ = codec.encode_batch_host(h_src, spans, order, h_enc)
        codec.decode_batch_host(h_enc, es, spans, h_dec)
        return es

    es = e2e_step()
    assert np.array_equal(h_dec[:n_bytes], data[:n_bytes]), "e2e round trip mismatch"
    e2e_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(cs)
        es = e2e_step()
        b.record(cs)
        b.synchronize()
        e2e_ms += a.elapsed_time(b)
    t = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_ms = float(t[0])
    cb = int(es[:, 1].sum())
    e2e = {"value": round(world * n_bytes * args.steps / (e2e_ms * 1e-3) / 1e9, 4), "unit": "GB/s",
           "h2d_bytes_per_step": (0 if decode_only else n_bytes) + cb,
           "d2h_bytes_per_step": (0 if decode_only else cb) + n_bytes,
           "path": "fqxv_rans_encode_batch_host + fqxv_rans_decode_batch_host (pinned host buffers)"}

    # ---- CPU baseline (rank 0, N = 1) -----------------------------------------
    cpu = None
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        from oracle import oracle

        nthreads = os.cpu_count() or 1
        if decode_only:
            def cstep():
                oracle.decode_batch(arena, enc_spans[:, 0], enc_spans[:, 1], spans[:, 1], nthreads)
        else:
            def cstep():
                oracle_roundtrip(data, spans, order, nthreads)
        cstep()
        t0 = time.perf_counter()
        reps = 0
        while True:
            cstep()
            reps += 1
            if time.perf_counter() - t0 > 5.0 or reps >= 20:
                break
        dt = time.perf_counter() - t0
        cpu = {"value": round(n_bytes * reps / dt / 1e9, 4), "unit": "GB/s", "cores": nthreads, "kind": "port",
               "sample": "%d passes of the whole workload (C restatement of fqxv-rans CPU path: AVX-512/AVX2 "
                         "order-0, scalar order-1), block-parallel over %d host threads" % (reps, nthreads)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": dict({"workload": args.workload, "desc": desc, "blocks": int(len(spans)),
                            "bytes_per_gpu": n_bytes, "compressed_bytes_per_gpu": comp_bytes,
                            "l2": "flushed (256 MiB write) before every timed step",
                            "parallelism": "replicas" if world > 1 else "single GPU"}, **extra),
            "encode_gbs": None if decode_only else round(world * n_bytes * args.steps / (enc_ms * 1e-3) / 1e9, 4),
            "decode_gbs": round(world * n_bytes * args.steps / (dec_ms * 1e-3) / 1e9, 4),
            "plain_per_block": plain,
            "byte_identical_blocks": identity["blocks"] if identity else None,
            "identity": identity,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": gpu_launches,
            "stages": {k: dict({"launches": v["launches"], "ms": round(v["ms"], 4), "wall_ms": round(v["wall_ms"], 4),
                                "bytes": v["bytes"]},
                               **({"ctas_per_sm": v["ctas_per_sm"], "smem_bytes": v["smem_bytes"]}
                                  if v.get("ctas_per_sm") else {}))
                       for k, v in stages.items() if v["launches"]},
            "clocks": clocks,
        }
    codec.close()
    if rank == 0 and world == 1 and args.serving_requests > 0 and args.workload == "config2":
        # a short serving pass (config4's loop) after the batch measurements
        line["serving"] = serving_levels(args.seed, args.serving_requests, [0.5, 1.0], args.workers)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
