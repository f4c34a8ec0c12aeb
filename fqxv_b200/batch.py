"""Batched device API: many independent blocks per GPU pass.

The reference codes container blocks independently on rayon workers
(crates/fqxv/src/container/compress.rs:868, decompress.rs:46-52). Here a whole
batch is one pass of the persistent kernels; device memory comes from torch
(plumbing only), the coding from libfqxv_rans_gpu.so.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import rans


class StageStat(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 24), ("launches", ctypes.c_uint64), ("ms", ctypes.c_double),
                ("bytes", ctypes.c_uint64), ("wall_ms", ctypes.c_double),
                ("ctas_per_sm", ctypes.c_uint32), ("smem_bytes", ctypes.c_uint32)]


# format.rs:252-266 StreamLoc, as include/fqxv_frame_gpu.h lays it out.
STREAM_LOC = np.dtype([("offset", "<u8"), ("len", "<u4"), ("crc", "<u4")])
# Frame statuses (include/fqxv_frame_gpu.h): per-frame results, not call failures.
FRAME_STATUSES = {32, 33, 34, 35}


def _spans(a) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(a, dtype=np.uint64).reshape(-1, 2))
    return a


class Codec:
    """One fqxv_rans_ctx: a CUDA stream plus device arenas on one GPU."""

    def __init__(self, device: int = 0):
        self._lib = rans.lib()
        h = ctypes.c_void_p()
        rans.raise_for(self._lib.fqxv_rans_ctx_create(device, ctypes.byref(h)))
        self._h = h
        self.device = device

    def close(self) -> None:
        if self._h:
            self._lib.fqxv_rans_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream_handle(self) -> int:
        return self._lib.fqxv_rans_ctx_stream(self._h)

    def device_bytes(self) -> int:
        return self._lib.fqxv_rans_ctx_device_bytes(self._h)

    def encode_bound(self, spans, order: int) -> int:
        s = _spans(spans)
        return self._lib.fqxv_rans_encode_batch_bound(s.ctypes.data, len(s), int(order))

    def encode_batch(self, d_src, spans, order: int, d_dst=None, persistent: bool = True):
        """Encode blocks `spans` (host (n, 2) offset/length) of the device
        tensor `d_src`. Returns (d_dst, out_spans, orders): the streams are
        back to back in d_dst in block order."""
        import torch

        s = _spans(spans)
        nb = len(s)
        if d_dst is None:
            d_dst = torch.empty(max(self.encode_bound(s, order), 1), dtype=torch.uint8, device=d_src.device)
        out = np.zeros((nb, 2), dtype=np.uint64)
        orders = np.zeros(nb, dtype=np.int32)
        st = self._lib.fqxv_rans_encode_batch(self._h, d_src.data_ptr(), s.ctypes.data, nb, int(order),
                                              d_dst.data_ptr(), d_dst.numel(), out.ctypes.data,
                                              orders.ctypes.data, 1 if persistent else 0)
        rans.raise_for(st)
        return d_dst, out, orders

    def decode_batch(self, d_src, spans, out_spans, max_len: int | None = None, d_dst=None,
                     persistent: bool = True, raise_on_error: bool = True):
        """Decode streams `spans` of d_src into d_dst at out_spans (offset,
        capacity). Returns (d_dst, out_lens, status). With raise_on_error
        False, per-stream statuses (malformed streams, and device waits that
        timed out) come back in `status` instead of raising."""
        import torch

        s = _spans(spans)
        o = _spans(out_spans)
        nb = len(s)
        if d_dst is None:
            need = int((o[:, 0] + o[:, 1]).max()) if nb else 1
            d_dst = torch.empty(max(need, 1), dtype=torch.uint8, device=d_src.device)
        lens = np.zeros(nb, dtype=np.uint64)
        status = np.zeros(nb, dtype=np.int32)
        ml = (1 << 64) - 1 if max_len is None else int(max_len)
        st = self._lib.fqxv_rans_decode_batch(self._h, d_src.data_ptr(), s.ctypes.data, nb, ml,
                                              d_dst.data_ptr(), o.ctypes.data, lens.ctypes.data,
                                              status.ctypes.data, 1 if persistent else 0)
        if st and (raise_on_error or st not in rans.STREAM_STATUSES):
            rans.raise_for(st)
        return d_dst, lens, status

    # ---- host-buffer batch forms ------------------------------------------

    def encode_batch_host(self, h_src: np.ndarray, spans, order: int, h_dst: np.ndarray):
        """Encode blocks of a host arena (pinned for DMA speed) into h_dst."""
        s = _spans(spans)
        nb = len(s)
        out = np.zeros((nb, 2), dtype=np.uint64)
        orders = np.zeros(nb, dtype=np.int32)
        st = self._lib.fqxv_rans_encode_batch_host(self._h, h_src.ctypes.data, s.ctypes.data, nb, int(order),
                                                   h_dst.ctypes.data, h_dst.size, out.ctypes.data,
                                                   orders.ctypes.data)
        rans.raise_for(st)
        return out, orders

    def decode_batch_host(self, h_src: np.ndarray, spans, out_spans, h_dst: np.ndarray,
                          max_len: int | None = None, raise_on_error: bool = True):
        s = _spans(spans)
        o = _spans(out_spans)
        nb = len(s)
        lens = np.zeros(nb, dtype=np.uint64)
        status = np.zeros(nb, dtype=np.int32)
        ml = (1 << 64) - 1 if max_len is None else int(max_len)
        st = self._lib.fqxv_rans_decode_batch_host(self._h, h_src.ctypes.data, s.ctypes.data, nb, ml,
                                                   h_dst.ctypes.data, o.ctypes.data, lens.ctypes.data,
                                                   status.ctypes.data)
        if st and (raise_on_error or st not in rans.MALFORMED):
            rans.raise_for(st)
        return lens, status

    # ---- CRC-32C and block frames (include/fqxv_frame_gpu.h) --------------

    def crc32c_batch(self, d_src, spans) -> np.ndarray:
        """CRC-32C (crates/fqxv/src/crc.rs:74) of each span of the device
        tensor d_src."""
        s = _spans(spans)
        out = np.zeros(len(s), dtype=np.uint32)
        rans.raise_for(self._lib.fqxv_crc32c_batch(self._h, d_src.data_ptr(), s.ctypes.data, len(s),
                                                   out.ctypes.data))
        return out

    def crc32c_batch_host(self, h_src: np.ndarray, spans) -> np.ndarray:
        s = _spans(spans)
        out = np.zeros(len(s), dtype=np.uint32)
        rans.raise_for(self._lib.fqxv_crc32c_batch_host(self._h, h_src.ctypes.data, s.ctypes.data, len(s),
                                                        out.ctypes.data))
        return out

    def frame_bound(self, spans, terminate: bool = False) -> int:
        s = _spans(spans)
        return self._lib.fqxv_frame_blocks_bound(s.ctypes.data, len(s), 1 if terminate else 0)

    def frame_blocks(self, d_src, spans, terminate: bool = False, d_dst=None):
        """Frame the payloads `spans` of d_src back to back
        (crates/fqxv/src/container/block.rs:110-142). Returns (d_dst,
        frame_offsets, crcs, total)."""
        import torch

        s = _spans(spans)
        need = self.frame_bound(s, terminate)
        if d_dst is None:
            d_dst = torch.empty(max(need, 1), dtype=torch.uint8, device=d_src.device)
        offs = np.zeros(len(s), dtype=np.uint64)
        crcs = np.zeros(len(s), dtype=np.uint32)
        tot = ctypes.c_uint64(0)
        rans.raise_for(self._lib.fqxv_frame_blocks(self._h, d_src.data_ptr(), s.ctypes.data, len(s),
                                                   1 if terminate else 0, d_dst.data_ptr(), d_dst.numel(),
                                                   offs.ctypes.data, crcs.ctypes.data, ctypes.byref(tot)))
        return d_dst, offs, crcs, tot.value

    def frame_blocks_host(self, h_src: np.ndarray, spans, h_dst: np.ndarray, terminate: bool = False):
        s = _spans(spans)
        offs = np.zeros(len(s), dtype=np.uint64)
        crcs = np.zeros(len(s), dtype=np.uint32)
        tot = ctypes.c_uint64(0)
        rans.raise_for(self._lib.fqxv_frame_blocks_host(self._h, h_src.ctypes.data, s.ctypes.data, len(s),
                                                        1 if terminate else 0, h_dst.ctypes.data, h_dst.size,
                                                        offs.ctypes.data, crcs.ctypes.data, ctypes.byref(tot)))
        return offs, crcs, tot.value

    def _read(self, fn, ptr, length: int, max_frames: int | None):
        cap = length // 16 + 1 if max_frames is None else int(max_frames)
        cap = min(cap, length // 16 + 1)
        pay = np.zeros((max(cap, 1), 2), dtype=np.uint64)
        crcs = np.zeros(max(cap, 1), dtype=np.uint32)
        status = np.zeros(max(cap, 1), dtype=np.int32)
        nf = ctypes.c_size_t(0)
        consumed = ctypes.c_uint64(0)
        term = ctypes.c_int(0)
        st = fn(self._h, ptr, length, cap, pay.ctypes.data, crcs.ctypes.data, status.ctypes.data, ctypes.byref(nf),
                ctypes.byref(consumed), ctypes.byref(term))
        if st and st not in FRAME_STATUSES:
            rans.raise_for(st)
        k = nf.value
        return pay[:k], crcs[:k], status[:k], consumed.value, bool(term.value)

    def read_blocks(self, d_src, length: int | None = None, max_frames: int | None = None):
        """Walk the frames of the device tensor d_src[:length]
        (block.rs:1209-1254, frame after frame) and verify every payload's
        CRC-32C. Returns (payload spans, crcs, status, consumed, terminated)."""
        n = d_src.numel() if length is None else int(length)
        return self._read(self._lib.fqxv_read_blocks, d_src.data_ptr(), n, max_frames)

    def read_blocks_host(self, h_src: np.ndarray, length: int | None = None, max_frames: int | None = None):
        n = h_src.size if length is None else int(length)
        return self._read(self._lib.fqxv_read_blocks_host, h_src.ctypes.data, n, max_frames)

    def payload_stream_locs(self, d_src, spans, base: int = 0):
        """block.rs:961-980 for each plain payload `spans` of d_src: an (n, 3)
        array of (offset, len, crc) stream locations and per-payload status."""
        s = _spans(spans)
        locs = np.zeros((len(s), 3), dtype=STREAM_LOC)
        status = np.zeros(len(s), dtype=np.int32)
        st = self._lib.fqxv_payload_stream_locs(self._h, d_src.data_ptr(), s.ctypes.data, len(s), int(base),
                                                locs.ctypes.data, status.ctypes.data)
        if st and st not in FRAME_STATUSES:
            rans.raise_for(st)
        return locs, status

    # ---- extended stream format (include/fqxv_rans_x_gpu.h) ----------------

    def _x_setup(self):
        L = self._lib
        if not getattr(L, "_x_ready", False):
            vp = ctypes.c_void_p
            L.fqxv_rans_x_encode_bound.restype = ctypes.c_uint64
            L.fqxv_rans_x_encode_bound.argtypes = [vp, ctypes.c_size_t]
            L.fqxv_rans_x_encode_batch.argtypes = [vp, vp, vp, ctypes.c_size_t, ctypes.c_int, vp, ctypes.c_uint64,
                                                   vp, vp]
            L.fqxv_rans_x_decode_batch.argtypes = [vp, vp, vp, ctypes.c_size_t, vp, vp, vp, vp]
            L._x_ready = True
        return L

    def x_encode_batch(self, d_src, spans, flags: int, d_dst=None):
        """Extended-format streams of the blocks `spans` of d_src with
        transform `flags` (or 0x40: the selection). Returns (d_dst,
        out_spans, choice)."""
        import torch

        L = self._x_setup()
        s = _spans(spans)
        nb = len(s)
        if d_dst is None:
            d_dst = torch.empty(max(L.fqxv_rans_x_encode_bound(s.ctypes.data, nb), 1), dtype=torch.uint8,
                                device=d_src.device)
        out = np.zeros((nb, 2), dtype=np.uint64)
        choice = np.zeros(nb, dtype=np.int32)
        rans.raise_for(L.fqxv_rans_x_encode_batch(self._h, d_src.data_ptr(), s.ctypes.data, nb, int(flags),
                                                  d_dst.data_ptr(), d_dst.numel(), out.ctypes.data,
                                                  choice.ctypes.data))
        return d_dst, out, choice

    def x_decode_batch(self, d_src, spans, out_spans, d_dst=None, raise_on_error: bool = True):
        """Decode extended (or reference) streams; returns (d_dst, out_lens, status)."""
        import torch

        L = self._x_setup()
        s = _spans(spans)
        o = _spans(out_spans)
        nb = len(s)
        if d_dst is None:
            need = int((o[:, 0] + o[:, 1]).max()) if nb else 1
            d_dst = torch.empty(max(need, 1), dtype=torch.uint8, device=d_src.device)
        lens = np.zeros(nb, dtype=np.uint64)
        status = np.zeros(nb, dtype=np.int32)
        st = L.fqxv_rans_x_decode_batch(self._h, d_src.data_ptr(), s.ctypes.data, nb, d_dst.data_ptr(),
                                        o.ctypes.data, lens.ctypes.data, status.ctypes.data)
        if st and (raise_on_error or st not in rans.STREAM_STATUSES):
            rans.raise_for(st)
        return d_dst, lens, status

    # ---- launch shapes (fqxv_rans_ctx_set_param) ----------------------------

    def set_param(self, name: str, value: int) -> None:
        L = self._lib
        L.fqxv_rans_ctx_set_param.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int64]
        rans.raise_for(L.fqxv_rans_ctx_set_param(self._h, name.encode(), int(value)))

    def get_param(self, name: str) -> int:
        L = self._lib
        L.fqxv_rans_ctx_get_param.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]
        v = ctypes.c_int64(0)
        rans.raise_for(L.fqxv_rans_ctx_get_param(self._h, name.encode(), ctypes.byref(v)))
        return int(v.value)

    def tuning_source(self) -> str:
        L = self._lib
        L.fqxv_rans_ctx_tuning_source.argtypes = [ctypes.c_void_p]
        L.fqxv_rans_ctx_tuning_source.restype = ctypes.c_char_p
        return L.fqxv_rans_ctx_tuning_source(self._h).decode()

    # ---- per-stage timing ---------------------------------------------------

    def set_profiling(self, on: bool) -> None:
        rans.raise_for(self._lib.fqxv_rans_ctx_set_profiling(self._h, 1 if on else 0))

    def stage_stats(self, reset: bool = False) -> dict:
        arr = (StageStat * 32)()
        n = ctypes.c_int(0)
        rans.raise_for(self._lib.fqxv_rans_ctx_stage_stats(self._h, ctypes.cast(arr, ctypes.c_void_p), 32,
                                                           ctypes.byref(n), 1 if reset else 0))
        return {arr[i].name.decode(): {"launches": int(arr[i].launches), "ms": float(arr[i].ms),
                                       "bytes": int(arr[i].bytes), "wall_ms": float(arr[i].wall_ms),
                                       "ctas_per_sm": int(arr[i].ctas_per_sm),
                                       "smem_bytes": int(arr[i].smem_bytes)}
                for i in range(n.value)}

    def _test_set_wait_polls(self, polls: int) -> None:
        """Test-only (include/fqxv_rans_gpu_testing.h): polls of a decode
        kernel's first wait for its table copy; 0 makes every staged stream
        report FQXV_RANS_E_TIMEOUT."""
        self._lib.fqxv_rans_ctx_test_set_wait_polls.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
        rans.raise_for(self._lib.fqxv_rans_ctx_test_set_wait_polls(self._h, int(polls)))
