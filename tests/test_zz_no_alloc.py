"""The no-allocation encode entry point (fqxv_rans_encode_noalloc).

It exists for callers that may not allocate device memory; its working memory
is a fixed device array inside the library. This test calls it through the C
ABI on device buffers the test owns and checks that its streams are identical
to those of the regular allocating entry point, call after call in one
process: every call shares the array and finds there whatever the previous
call left (tables, histogram, renorm words of either order), so a stale
leftover that reached a stream would show as a difference.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib, torch, data: bytes, order: int) -> bytes:
    fn = lib.fqxv_rans_encode_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t,
                   ctypes.POINTER(ctypes.c_size_t), ctypes.c_void_p]
    fn.restype = ctypes.c_int
    # a one-byte buffer stands in for the source of an empty input
    src = torch.from_numpy(np.frombuffer(data or b"\0", dtype=np.uint8).copy()).cuda()
    cap = lib.fqxv_rans_encode_bound(len(data), order)
    dst = torch.full((cap,), 0xA5, dtype=torch.uint8, device="cuda")
    out_len = ctypes.c_size_t(0)
    stream = torch.cuda.current_stream().cuda_stream
    rc = fn(src.data_ptr(), len(data), order, dst.data_ptr(), cap, ctypes.byref(out_len), stream)
    assert rc == 0, rc
    torch.cuda.synchronize()
    return dst[:out_len.value].cpu().numpy().tobytes()


def test_noalloc_matches_allocating_entry_point_call_after_call():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from fqxv_b200 import rans, workloads

    lib = rans.lib()
    wide = workloads.full_quality(1 << 20, seed=21).tobytes()        # order-1, a wide alphabet, the maximum size
    small = workloads.binned_quality(70_001, seed=22).tobytes()      # a 5-symbol alphabet, shorter
    names = workloads.GENERATORS["names"](300_000, 23).tobytes()
    calls = [
        (wide, 1),
        (small, 1),     # order-1 after order-1: the wide call's tables, histogram and words are still there
        (small, 0),
        (names, 2),     # BEST_TIE0: both orders' word regions in one call
        (wide[:200_000], 3),   # BEST_TIE1
        (small[:5_000], 2),
        (b"", 0),       # n = 0: the 9-byte stream, for every mode
        (b"", 1),
        (b"", 2),
        (b"", 3),
        (small[:1], 1),
        (wide, 1),      # the first call again, after everything else
    ]
    for data, order in calls:
        got = _noalloc(lib, torch, data, order)
        want = rans.encode(data, rans.Order(order))
        assert got == want, "no-alloc stream differs from the allocating entry point (n=%d, mode %d)" % (
            len(data), order)
    # inputs above the stated maximum are refused, not truncated
    big = torch.zeros((1 << 20) + 1, dtype=torch.uint8, device="cuda")
    out = torch.zeros(16, dtype=torch.uint8, device="cuda")
    n = ctypes.c_size_t(0)
    rc = lib.fqxv_rans_encode_noalloc(big.data_ptr(), big.numel(), 0, out.data_ptr(), 16, ctypes.byref(n),
                                      torch.cuda.current_stream().cuda_stream)
    assert rc == 22
