"""Seeded synthetic inputs with the shapes of the benchmark configurations.

There is no public dataset for this path; every generator below is seeded
numpy. Each returns an input arena (u8) and block spans (offset, length).

* binned_quality  -- Illumina binned quality: '#', ',', ':', 'F' with
  p = 0.02 / 0.05 / 0.13 / 0.80; each symbol repeats the previous one with
  p = 0.7, otherwise redraws; 151-byte reads concatenated.
* full_quality    -- 150 positions per read, Q = clamp(round(N(38 - 0.08 pos,
  3)), 2, 41) + 33; 1% of reads end in a run of Q2 starting at a uniform
  position in 0..149.
* acgt            -- uniform A/C/G/T with 0.1% N.
* name_tokens     -- ASCII decimal fields of uniform u16 integers plus
  delta-coded tile / x / y fields, ':'-separated, one record per line.
* ont_quality     -- long reads, length log-normal (median 8000, sigma 0.8),
  per-read mean U(10, 25), per-base N(mean, 6) clamped to Q3..Q40, +33.
* quality_like    -- the reference benchmark's xorshift random walk over
  Q2..Q41 (crates/fqxv-rans/benches/rans.rs:11-25).
"""

from __future__ import annotations

import numpy as np

MiB = 1 << 20
KiB = 1 << 10


def binned_quality(n: int, seed: int = 0, read_len: int = 151) -> np.ndarray:
    rng = np.random.default_rng(seed)
    alphabet = np.frombuffer(b"#,:F", dtype=np.uint8)
    draws = alphabet[rng.choice(4, size=n, p=[0.02, 0.05, 0.13, 0.80])]
    repeat = rng.random(n) < 0.7
    repeat[::read_len] = False  # first base of every read is a fresh draw
    idx = np.where(repeat, 0, np.arange(n))
    np.maximum.accumulate(idx, out=idx)
    return draws[idx]


def full_quality(n: int, seed: int = 0, read_len: int = 150) -> np.ndarray:
    rng = np.random.default_rng(seed)
    nreads = -(-n // read_len)
    pos = np.arange(read_len, dtype=np.float64)
    q = np.rint(rng.normal(38.0 - 0.08 * pos, 3.0, size=(nreads, read_len)))
    q = np.clip(q, 2, 41)
    tail = rng.random(nreads) < 0.01
    starts = rng.integers(0, read_len, size=nreads)
    mask = tail[:, None] & (pos[None, :] >= starts[:, None])
    q[mask] = 2
    return (q.astype(np.uint8) + 33).reshape(-1)[:n]


def acgt(n: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    out = np.frombuffer(b"ACGT", dtype=np.uint8)[rng.integers(0, 4, size=n)]
    out = out.copy()
    out[rng.random(n) < 0.001] = ord("N")
    return out


def _ascii_ints(v: np.ndarray, width: int = 7) -> np.ndarray:
    """Decimal text of signed integers (|v| < 10**(width-1)) as a (k, width)
    byte matrix, right-aligned, with 0 in the unused leading cells."""
    neg = v < 0
    a = np.abs(v).astype(np.int64)
    out = np.zeros((len(v), width), dtype=np.uint8)
    nd = np.ones(len(v), dtype=np.int64)
    t = a.copy()
    for col in range(width - 1, -1, -1):
        out[:, col] = 48 + (t % 10)
        t //= 10
    x = a.copy()
    while True:
        x //= 10
        more = x > 0
        if not more.any():
            break
        nd += more
    lead = width - nd
    cols = np.arange(width)[None, :]
    out[cols < lead[:, None]] = 0
    sign_col = lead - 1
    rows = np.nonzero(neg)[0]
    out[rows, sign_col[rows]] = ord("-")
    return out


def name_tokens(n: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    k = n // 12 + 16
    fields = [
        rng.integers(0, 65536, size=k),                 # uniform u16 fields
        rng.integers(0, 65536, size=k),
        (rng.random(k) < 0.01).astype(np.int64),        # tile delta
        rng.integers(0, 40, size=k),                    # x delta
        rng.integers(-2000, 2000, size=k),              # y delta
    ]
    cols = []
    for j, f in enumerate(fields):
        cols.append(_ascii_ints(f))
        sep = np.full((k, 1), ord(":") if j < len(fields) - 1 else ord("\n"), dtype=np.uint8)
        cols.append(sep)
    mat = np.concatenate(cols, axis=1).reshape(-1)
    text = mat[mat != 0]
    while len(text) < n:
        text = np.concatenate([text, text])
    return text[:n].copy()


def ont_reads(nreads: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    lens = np.maximum(1, rng.lognormal(np.log(8000.0), 0.8, size=nreads).astype(np.int64))
    means = rng.uniform(10, 25, size=nreads)
    per_base = np.repeat(means, lens)
    q = np.clip(np.rint(rng.normal(per_base, 6.0)), 3, 40).astype(np.uint8) + 33
    return q


def quality_like(n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.uint8)
    state = 0x12345678
    q = 30
    for i in range(n):
        state ^= (state << 13) & 0xFFFFFFFF
        state ^= state >> 17
        state ^= (state << 5) & 0xFFFFFFFF
        step = (state % 7) - 3
        q = min(max(q + step, 2), 41)
        out[i] = 33 + q
    return out


GENERATORS = {"binned": binned_quality, "full": full_quality, "acgt": acgt, "names": name_tokens}


def _spans(lengths) -> np.ndarray:
    lengths = np.asarray(lengths, dtype=np.uint64)
    offs = np.zeros(len(lengths), dtype=np.uint64)
    if len(lengths):
        offs[1:] = np.cumsum(lengths)[:-1]
    return np.stack([offs, lengths], axis=1)


def config0(total: int = MiB, seed: int = 0):
    """One binned-quality block, order-0."""
    data = binned_quality(total, seed)
    return data, _spans([total])


def config1(nblocks: int = 64, block: int = MiB, seed: int = 0):
    """Full-range quality cut into equal blocks, order-1."""
    data = full_quality(nblocks * block, seed)
    return data, _spans([block] * nblocks)


def _gen_one(args):
    name, size, seed = args
    return GENERATORS[name](size, seed)


def uniform_batch(kind: str, nblocks: int = 2048, block: int = 512 * KiB, seed: int = 0):
    """Many equal blocks of one stream type (binned or full-range quality):
    the shape for peak batched throughput of one order and direction."""
    gen = binned_quality if kind == "binned" else full_quality
    data = gen(nblocks * block, seed)
    return data, _spans([block] * nblocks)


def config2(nblocks: int = 4096, lo: int = 4 * KiB, hi: int = 4 * MiB, seed: int = 0, workers: int = 0):
    """Mixed blocks, sizes log-uniform in [lo, hi], stream type uniform over
    the four generators; block i is seeded with seed + i. `workers` > 1
    generates blocks in a spawn-started process pool (the output is the same)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), size=nblocks)).astype(np.int64)
    kinds = rng.integers(0, 4, size=nblocks)
    names = list(GENERATORS)
    jobs = [(names[k], int(s), seed + i) for i, (s, k) in enumerate(zip(sizes, kinds))]
    if workers > 1 and nblocks > 64:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor

        with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            blocks = list(ex.map(_gen_one, jobs, chunksize=16))
    else:
        blocks = [_gen_one(j) for j in jobs]
    data = np.concatenate(blocks) if blocks else np.zeros(0, np.uint8)
    return data, _spans(sizes), [names[k] for k in kinds]


def config3_ont(nreads: int = 2000, lo: int = 256 * KiB, hi: int = 8 * MiB, seed: int = 0):
    """ONT-like quality packed into blocks cut at log-uniform sizes."""
    data = ont_reads(nreads, seed)
    rng = np.random.default_rng(seed + 1)
    sizes = []
    left = len(data)
    while left > 0:
        s = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        s = min(s, left)
        sizes.append(s)
        left -= s
    return data, _spans(sizes)
