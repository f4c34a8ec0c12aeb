"""The no-allocation encode entry point (fqxv_rans_encode_noalloc).

It exists for callers that may not allocate device memory; its working memory
is a fixed device array inside the library. This test calls it through the C
ABI on device buffers the test owns and checks that its streams are identical
to those of the regular allocating entry point, on two calls in a row (the
second call must not see anything the first one left in the shared array).
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
    src = torch.from_numpy(np.frombuffer(data, dtype=np.uint8).copy()).cuda()
    cap = lib.fqxv_rans_encode_bound(len(data), order)
    dst = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    out_len = ctypes.c_size_t(0)
    stream = torch.cuda.current_stream().cuda_stream
    rc = fn(src.data_ptr(), len(data), order, dst.data_ptr(), cap, ctypes.byref(out_len), stream)
    assert rc == 0, rc
    torch.cuda.synchronize()
    return dst[:out_len.value].cpu().numpy().tobytes()


def test_noalloc_matches_allocating_entry_point_twice_in_a_row():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from fqxv_b200 import rans, workloads

    lib = rans.lib()
    first = workloads.full_quality(1 << 20, seed=21).tobytes()        # order-1, a wide alphabet
    second = workloads.binned_quality(70_001, seed=22).tobytes()      # smaller, order-0
    for data, order in ((first, 1), (second, 0)):
        got = _noalloc(lib, torch, data, order)
        want = rans.encode(data, rans.Order(order))
        assert got == want, "no-alloc stream differs from the allocating entry point (order %d)" % order
    # inputs above the stated maximum are refused, not truncated
    big = torch.zeros((1 << 20) + 1, dtype=torch.uint8, device="cuda")
    out = torch.zeros(16, dtype=torch.uint8, device="cuda")
    n = ctypes.c_size_t(0)
    rc = lib.fqxv_rans_encode_noalloc(big.data_ptr(), big.numel(), 0, out.data_ptr(), 16, ctypes.byref(n),
                                      torch.cuda.current_stream().cuda_stream)
    assert rc == 22
