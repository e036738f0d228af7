"""The allocation-free prefix sum (gsr_prefix_sum_u32_noalloc).

It serves callers that cannot let a library allocate device memory, for
example frameworks that own the device's memory budget through their own
pool. The test calls it through the C ABI, two calls in a row per pair of
lengths (the second with different data and a different length, so stale
scratch from the first would show), and checks each result exactly, as an
integer scan must be, against the host's np.cumsum in uint32 (which wraps
modulo 2^32 as the device scan does) and against the regular context-based
scan, gsr_prefix_sum_u32. The lengths include the documented maximum 2^24,
where every one of the 8,192 look-back states is in use, and 2^24 - 1, which
ends in a partial partition. It also checks that a length above the maximum
is refused before any device work."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lengths", [(3_000_001, 1_048_576), (1 << 24, (1 << 24) - 1)])
def test_noalloc_prefix_sum_matches_host_and_context_scan(lengths):
    import torch

    from rustscan_b200 import Context, _lib

    L = _lib.load()
    ctx = Context(max_splats=1 << 20)
    rng = np.random.default_rng(123 + lengths[0])
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for n in lengths:
        # Values up to 2^10: sums past 2^32 at the largest lengths, so the
        # wrap-around is exercised too.
        x_np = rng.integers(0, 1 << 10, n, dtype=np.uint32)
        x = torch.as_tensor(x_np.view(np.int32), device="cuda")
        out = torch.full_like(x, -1)
        st = L.gsr_prefix_sum_u32_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()), n, stream)
        assert st == _lib.GSR_OK
        ref = ctx.prefix_sum_u32(x)
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(np.uint32)
        np.testing.assert_array_equal(got, np.cumsum(x_np, dtype=np.uint32))
        np.testing.assert_array_equal(got, ref.cpu().numpy().view(np.uint32))
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
    assert st == _lib.GSR_ERR_INVALID_ARG
