"""Scan and sort primitives through the C ABI against the reference's known
answers (gpu_primitives/{prefix_sum,radix_sort}/tests.rs) and numpy."""
import json
import time
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_known_answers.json")))


@pytest.fixture(scope="module")
def ctx(gsr_ctx_factory):
    return gsr_ctx_factory(max_splats=1 << 22, max_isects=1 << 22)


def _t(a):
    import torch

    return torch.as_tensor(np.asarray(a, dtype=np.uint32).view(np.int32), device="cuda")


def _np(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("case", GOLD["prefix_sum"], ids=lambda c: c["test"])
def test_prefix_sum_known_answers(ctx, case):
    out = ctx.prefix_sum_u32(_t(case["input"]))
    np.testing.assert_array_equal(_np(out), np.asarray(case["expected"], np.uint32))


@pytest.mark.parametrize("case", GOLD["argsort"], ids=lambda c: c["test"])
def test_argsort_known_answers(ctx, case):
    keys = case["keys"]
    _, vals = ctx.radix_sort_by_key_u32(_t(keys), _t(np.arange(len(keys))))
    np.testing.assert_array_equal(_np(vals), np.asarray(case["expected"], np.uint32))


def test_sort_by_key_known_answer(ctx):
    c = GOLD["sort_by_key"][0]
    k, v = ctx.radix_sort_by_key_u32(_t(c["keys"]), _t(c["values"]))
    np.testing.assert_array_equal(_np(k), np.asarray(c["expected_keys"], np.uint32))
    np.testing.assert_array_equal(_np(v), np.asarray(c["expected_values"], np.uint32))


@pytest.mark.parametrize("n", [1, 7, 255, 256, 257, 2047, 2048, 2049, 100_003, 3_000_000])
def test_prefix_sum_random(ctx, n):
    rng = np.random.default_rng(n)
    x = rng.integers(0, 50, n, dtype=np.uint32)
    out = _np(ctx.prefix_sum_u32(_t(x)))
    np.testing.assert_array_equal(out, np.cumsum(x, dtype=np.uint64).astype(np.uint32))


@pytest.mark.parametrize("n,kmax", [(1, 10), (33, 4), (4095, 1 << 32), (4096, 7), (4097, 1 << 20), (250_000, 1 << 32),
                                    (2_000_000, 300), (4_000_000, 1 << 32)])
def test_sort_random_stable(ctx, n, kmax):
    rng = np.random.default_rng(n + 1)
    keys = rng.integers(0, kmax, n, dtype=np.uint64).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    k, v = ctx.radix_sort_by_key_u32(_t(keys), _t(vals))
    order = np.argsort(keys, kind="stable").astype(np.uint32)
    np.testing.assert_array_equal(_np(v), order)
    np.testing.assert_array_equal(_np(k), keys[order])


def test_sort_repeat_is_deterministic(ctx):
    rng = np.random.default_rng(5)
    keys = rng.integers(0, 1000, 1_000_000, dtype=np.uint32)
    a = _np(ctx.radix_sort_by_key_u32(_t(keys), _t(np.arange(keys.size)))[1])
    b = _np(ctx.radix_sort_by_key_u32(_t(keys), _t(np.arange(keys.size)))[1])
    np.testing.assert_array_equal(a, b)


def test_bounded_wait_gives_up_and_context_stays_usable(ctx):
    """A look-back whose predecessor never publishes (a flag nothing sets)
    gives up after its poll limit and reports GSR_ERR_TIMEOUT with the wait
    site; no fault, no hang, and the context keeps working afterwards."""
    import ctypes as C

    import torch

    t0 = time.perf_counter()
    st = ctx._lib.gsr_selftest_wait_timeout(ctx._h, 1 << 14, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    dt = time.perf_counter() - t0
    assert st == 5, st
    assert b"bounded device wait gave up (site 4)" in ctx._lib.gsr_last_error(ctx._h)
    assert dt < 10.0
    # A scan (look-back) right after works and is exact.
    x = np.arange(5000, dtype=np.uint32) % 7
    out = ctx.prefix_sum_u32(_t(x))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), np.cumsum(x, dtype=np.uint32))
    ctx.sync_status()

