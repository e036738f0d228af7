"""The allocation-free prefix sum (gsr_prefix_sum_u32_noalloc).

It serves callers that cannot let a library allocate device memory, for
example frameworks that own the device's memory budget through their own
pool. The test calls it through the C ABI and compares it with the regular
context-based scan, gsr_prefix_sum_u32, on two calls in a row (the second
with different data and a different length, so stale scratch from the
first would show). Integer scans must agree exactly. It also checks that a
length above the fixed 2^24 limit is refused."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_prefix_sum_matches_context_scan():
    import torch

    from rustscan_b200 import Context, _lib

    L = _lib.load()
    ctx = Context(max_splats=1 << 20)
    rng = np.random.default_rng(123)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for n in (3_000_001, 1_048_576):
        x = torch.as_tensor(rng.integers(0, 1000, n, dtype=np.uint32).view(np.int32), device="cuda")
        out = torch.full_like(x, -1)
        st = L.gsr_prefix_sum_u32_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()), n, stream)
        assert st == _lib.GSR_OK
        ref = ctx.prefix_sum_u32(x)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), ref.cpu().numpy())
    ctx.close()


def test_noalloc_prefix_sum_rejects_oversized_input():
    import torch

    from rustscan_b200 import _lib

    L = _lib.load()
    x = torch.zeros(16, dtype=torch.int32, device="cuda")
    y = torch.zeros(16, dtype=torch.int32, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    # The length check runs before any device work, so the small buffers are never touched.
    st = L.gsr_prefix_sum_u32_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), (1 << 24) + 1, stream)
    assert st == 1  # GSR_ERR_INVALID_ARG, before any device work
