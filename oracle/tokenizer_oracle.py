"""CPU restatement of the read-name tokenizer -- TEST INFRASTRUCTURE ONLY.

Follows `crates/fqxv-tokenizer/src/lib.rs` (encode :482-540, decode :543-650,
tokenize :654-680, num_tok :684-699, the stream helpers :91-254, constants
:54-75) and the varint / zigzag helpers of `crates/fqxv-bytes/src/lib.rs`
(:14-60, Reader :131-150), over the C oracle's rANS coder. Errors are raised as
`TokError(message)` with the reference's `Error::Malformed` text, or
`oracle.OracleError` for the rANS errors the reference passes through.

Pinned by the four names payloads the reference stored in its golden archives
(`tests/golden/fixture_names.*`): decoding each and re-encoding the names
reproduces the stored bytes exactly.
"""

from __future__ import annotations

from . import oracle

FORMAT_VERSION = 1
MATCH, STR, NUM, DELTA = 0, 1, 2, 3
MAX_NUM_DIGITS = 18
MAX_COL = 63
MAX_STREAM_EXPANSION = 1 << 16
MIN_STREAM_BOUND = 1 << 20
M64 = (1 << 64) - 1


class TokError(Exception):
    def __init__(self, message: str):
        super().__init__("malformed name stream: " + message)
        self.message = message


def write_varint(out: bytearray, v: int) -> None:
    v &= M64
    while True:
        b = v & 0x7F
        v >>= 7
        if v == 0:
            out.append(b)
            return
        out.append(b | 0x80)


class Reader:
    """fqxv-bytes Reader with the tokenizer's errors (lib.rs:700-711)."""

    def __init__(self, buf: bytes):
        self.buf = buf
        self.pos = 0

    def u8(self) -> int:
        if self.pos >= len(self.buf):
            raise TokError("truncated")
        self.pos += 1
        return self.buf[self.pos - 1]

    def varint(self) -> int:
        # fqxv-bytes read_varint (:32-47): any failure, truncation included, is
        # the reader's bad_varint ("varint too long"); bits past 64 drop.
        v = 0
        shift = 0
        while True:
            if self.pos >= len(self.buf):
                raise TokError("varint too long")
            b = self.buf[self.pos]
            self.pos += 1
            v |= ((b & 0x7F) << shift) & M64
            if b & 0x80 == 0:
                return v
            shift += 7
            if shift >= 64:
                raise TokError("varint too long")

    def take(self, n: int) -> bytes:
        if self.pos + n > len(self.buf):
            raise TokError("truncated")
        s = self.buf[self.pos:self.pos + n]
        self.pos += n
        return s


def zigzag(d: int) -> int:
    return ((d << 1) ^ (d >> 63)) & M64


def unzigzag(z: int) -> int:
    v = (z >> 1) ^ (-(z & 1))
    return to_i64(v)


def to_i64(v: int) -> int:
    v &= M64
    return v - (1 << 64) if v >> 63 else v


def natural_digits(value: int) -> int:
    return 1 if value <= 0 else len(str(value))


def tokenize(name: bytes):
    toks = []
    i = 0
    while i < len(name):
        d = 48 <= name[i] <= 57
        s = i
        while i < len(name) and (48 <= name[i] <= 57) == d:
            i += 1
        b = name[s:i]
        is_num = d and len(b) <= MAX_NUM_DIGITS
        toks.append((is_num, b, int(b) if is_num else 0))
    return toks


def num_tok(value: int, width: int):
    s = str(value).encode()
    if len(s) < width:
        s = b"0" * (width - len(s)) + s
    return (True, s, value)


def encode_best(stream: bytes) -> bytes:
    o0 = oracle.encode(stream, 0)
    o1 = oracle.encode(stream, 1)
    return o1 if len(o1) < len(o0) else o0


def push_stream(out: bytearray, stream: bytes) -> None:
    c = encode_best(bytes(stream))
    write_varint(out, len(c))
    out += c


def role_streams(names):
    """The role streams encode builds before coding (lib.rs:482-524)."""
    counts = bytearray()
    op_cols = [bytearray() for _ in range(MAX_COL + 1)]
    str_lens, str_data, num_vals, pads = bytearray(), bytearray(), bytearray(), bytearray()
    delta_vals = [[] for _ in range(MAX_COL + 1)]
    prev = []
    for name in names:
        toks = tokenize(bytes(name))
        for i, t in enumerate(toks):
            col = min(i, MAX_COL)
            p = prev[i] if i < len(prev) else None
            if p is not None and p[1] == t[1]:
                op_cols[col].append(MATCH)
            elif t[0]:
                pad = len(t[1]) - natural_digits(t[2])
                if p is not None and p[0]:
                    op_cols[col].append(DELTA)
                    delta_vals[col].append(zigzag(t[2] - p[2]))
                else:
                    op_cols[col].append(NUM)
                    write_varint(num_vals, t[2])
                pads.append(pad)
            else:
                op_cols[col].append(STR)
                write_varint(str_lens, len(t[1]))
                str_data += t[1]
        write_varint(counts, len(toks))
        prev = toks
    return counts, str_lens, str_data, num_vals, pads, op_cols, delta_vals


def op_rle(cols):
    """lib.rs:176-202."""
    counts, syms, lens = bytearray(), bytearray(), bytearray()
    for col in cols:
        runs = 0
        i = 0
        while i < len(col):
            s = col[i]
            r = 1
            while i + r < len(col) and col[i + r] == s:
                r += 1
            syms.append(s)
            write_varint(lens, r)
            runs += 1
            i += r
        write_varint(counts, runs)
    return counts, syms, lens


def delta_planes(cols):
    """lib.rs:118-137: per column [width, planes...] (width 0: empty)."""
    out = []
    for col in cols:
        if not col:
            out.append((0, []))
            continue
        m = max(col)
        width = max(1, (m.bit_length() + 7) // 8)
        out.append((width, [bytes((v >> (8 * p)) & 0xFF for v in col) for p in range(width)]))
    return out


def encode(names) -> bytes:
    counts, str_lens, str_data, num_vals, pads, op_cols, delta_vals = role_streams(names)
    out = bytearray([FORMAT_VERSION])
    write_varint(out, len(names))
    for s in (counts, str_lens, str_data, num_vals, pads):
        push_stream(out, s)
    for s in op_rle(op_cols):
        push_stream(out, s)
    for width, planes in delta_planes(delta_vals):
        write_varint(out, width)
        for p in planes:
            push_stream(out, p)
    return bytes(out)


def _decode_bounded(stream: bytes, bound: int) -> bytes:
    st, out = oracle.decode_status(stream, max_len=bound)
    if st:
        raise oracle.OracleError(st)
    return out


def decode(src: bytes) -> list[bytes]:
    """lib.rs:543-650."""
    r = Reader(src)
    if r.u8() != FORMAT_VERSION:
        raise TokError("unsupported version")
    n_records = r.varint()
    max_out = max(len(src) * MAX_STREAM_EXPANSION, MIN_STREAM_BOUND)

    def read_stream():
        ln = r.varint()
        return _decode_bounded(r.take(ln), max_out)

    counts = read_stream()
    if n_records > len(counts):
        raise TokError("record count exceeds token stream")
    str_lens = read_stream()
    str_data = read_stream()
    num_vals = read_stream()
    pads = read_stream()
    # read_op_rle (lib.rs:205-254)
    oc, osy, olen = read_stream(), read_stream(), read_stream()
    rc, rl = Reader(oc), Reader(olen)
    sym_pos = 0
    total = 0
    op_data = []
    for _ in range(MAX_COL + 1):
        n_runs = rc.varint()
        col = bytearray()
        for _ in range(n_runs):
            if sym_pos >= len(osy):
                raise TokError("op sym underrun")
            s = osy[sym_pos]
            sym_pos += 1
            run = rl.varint()
            if len(col) + run > n_records:
                raise TokError("op run too long")
            total += run
            if total > max_out:
                raise TokError("op columns exceed the stream bound")
            col += bytes([s]) * run
        op_data.append(bytes(col))
    n_delta = [sum(1 for o in col if o == DELTA) for col in op_data]
    # read_delta_planes (lib.rs:140-170)
    delta_vals = []
    for n in n_delta:
        width = r.varint()
        if width == 0:
            delta_vals.append([])
            continue
        vals = [0] * n
        for plane in range(width):
            ln = r.varint()
            b = _decode_bounded(r.take(ln), n)
            if len(b) != n:
                raise TokError("delta plane length mismatch")
            for i, x in enumerate(b):
                vals[i] |= x << (8 * plane)
        delta_vals.append([v & M64 for v in vals])

    ops = [Reader(c) for c in op_data]
    dpos = [0] * (MAX_COL + 1)
    c_counts, c_lens, c_num = Reader(counts), Reader(str_lens), Reader(num_vals)
    str_pos = 0
    pad_pos = 0
    names = []
    prev = []
    for _ in range(n_records):
        n_toks = c_counts.varint()
        cur = []
        for _ in range(n_toks):
            col = min(len(cur), MAX_COL)
            op = ops[col].u8()
            if op == MATCH:
                if len(cur) >= len(prev):
                    raise TokError("MATCH without prior token")
                cur.append(prev[len(cur)])
            elif op == STR:
                ln = c_lens.varint()
                if str_pos + ln > len(str_data):
                    raise TokError("string data underrun")
                cur.append((False, str_data[str_pos:str_pos + ln], 0))
                str_pos += ln
            elif op == NUM:
                value = to_i64(c_num.varint())
                if pad_pos >= len(pads):
                    raise TokError("pad underrun")
                width = natural_digits(value) + pads[pad_pos]
                pad_pos += 1
                cur.append(num_tok(value, width))
            elif op == DELTA:
                if dpos[col] >= len(delta_vals[col]):
                    raise TokError("delta underrun")
                z = delta_vals[col][dpos[col]]
                dpos[col] += 1
                d = unzigzag(z)
                p = prev[len(cur)] if len(cur) < len(prev) else None
                if p is None or not p[0]:
                    raise TokError("DELTA without numeric prior")
                value = to_i64(p[2] + d)
                if pad_pos >= len(pads):
                    raise TokError("pad underrun")
                width = natural_digits(value) + pads[pad_pos]
                pad_pos += 1
                cur.append(num_tok(value, width))
            else:
                raise TokError("unknown op")
        names.append(b"".join(t[1] for t in cur))
        prev = cur
    return names
