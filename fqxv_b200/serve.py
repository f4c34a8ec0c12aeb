"""Serving front end: continuous batching of compress / decompress requests
on one GPU (the C++ runtime in csrc/rans_server.cu).

    with Server(device=0, workers=8, hbm_cap=40 << 30) as srv:
        rid = srv.submit_encode(data, Order.One)
        stream = srv.result(rid)            # bytes, or raises Malformed
        lat_us = srv.last_latency_us

Requests are admitted in arrival order while their device-memory estimate fits
under `hbm_cap`; a free worker codes every admitted request of the oldest
request's kind, order mode and size class (within a factor of four) as one
batched pass.
"""

from __future__ import annotations

import ctypes

from . import rans

_bound = False


def _lib():
    global _bound
    L = rans.lib()
    if not _bound:
        vp = ctypes.c_void_p
        L.fqxv_rans_server_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(vp)]
        L.fqxv_rans_server_destroy.argtypes = [vp]
        L.fqxv_rans_server_destroy.restype = None
        L.fqxv_rans_server_submit.argtypes = [vp, ctypes.c_int, vp, ctypes.c_size_t, ctypes.c_int, ctypes.c_uint64,
                                              ctypes.POINTER(ctypes.c_uint64)]
        L.fqxv_rans_server_wait.argtypes = [vp, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t),
                                            ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double)]
        L.fqxv_rans_server_take.argtypes = [vp, ctypes.c_uint64, vp, ctypes.c_size_t]
        L.fqxv_rans_server_stats.argtypes = [vp] + [ctypes.POINTER(ctypes.c_uint64)] * 4
        _bound = True
    return L


class Server:
    def __init__(self, device: int = 0, workers: int = 8, hbm_cap: int = 40 << 30):
        self._L = _lib()
        h = ctypes.c_void_p()
        rans.raise_for(self._L.fqxv_rans_server_create(device, workers, hbm_cap, ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        if self._h:
            self._L.fqxv_rans_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _submit(self, kind: int, data, order: int, max_len: int) -> int:
        b = bytes(data)
        rid = ctypes.c_uint64(0)
        st = self._L.fqxv_rans_server_submit(self._h, kind, ctypes.cast(ctypes.c_char_p(b), ctypes.c_void_p),
                                             len(b), int(order), max_len, ctypes.byref(rid))
        rans.raise_for(st)
        return rid.value

    def submit_encode(self, data, order=rans.Order.Zero) -> int:
        return self._submit(0, data, int(order), 0)

    def submit_decode(self, data, max_len: int = (1 << 64) - 1) -> int:
        return self._submit(1, data, 0, max_len)

    def wait(self, rid: int, timeout_ms: int = -1):
        """-> (done, out_len, status, latency_us)."""
        n = ctypes.c_size_t(0)
        st = ctypes.c_int32(0)
        lat = ctypes.c_double(0)
        rc = self._L.fqxv_rans_server_wait(self._h, rid, timeout_ms, ctypes.byref(n), ctypes.byref(st),
                                           ctypes.byref(lat))
        if rc == 21:
            return False, 0, 0, 0.0
        rans.raise_for(rc)
        return True, n.value, st.value, lat.value

    def result(self, rid: int, timeout_ms: int = -1) -> bytes:
        done, n, st, lat = self.wait(rid, timeout_ms)
        if not done:
            raise TimeoutError("request %d not done" % rid)
        self.last_latency_us = lat
        buf = ctypes.create_string_buffer(max(n, 1))
        rans.raise_for(self._L.fqxv_rans_server_take(self._h, rid, buf, max(n, 1)))
        rans.raise_for(st)
        return buf.raw[:n]

    def stats(self) -> dict:
        v = [ctypes.c_uint64(0) for _ in range(4)]
        rans.raise_for(self._L.fqxv_rans_server_stats(self._h, *[ctypes.byref(x) for x in v]))
        return {"completed": v[0].value, "batches": v[1].value, "peak_bytes": v[2].value, "pending": v[3].value}
