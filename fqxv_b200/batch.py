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
                ("bytes", ctypes.c_uint64)]


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
        capacity). Returns (d_dst, out_lens, status)."""
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
        if st and (raise_on_error or st not in rans.MALFORMED):
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

    # ---- per-stage timing ---------------------------------------------------

    def set_profiling(self, on: bool) -> None:
        rans.raise_for(self._lib.fqxv_rans_ctx_set_profiling(self._h, 1 if on else 0))

    def stage_stats(self, reset: bool = False) -> dict:
        arr = (StageStat * 16)()
        n = ctypes.c_int(0)
        rans.raise_for(self._lib.fqxv_rans_ctx_stage_stats(self._h, ctypes.cast(arr, ctypes.c_void_p), 16,
                                                           ctypes.byref(n), 1 if reset else 0))
        return {arr[i].name.decode(): {"launches": int(arr[i].launches), "ms": float(arr[i].ms),
                                       "bytes": int(arr[i].bytes)} for i in range(n.value)}
