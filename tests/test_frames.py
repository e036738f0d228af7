"""Frame pipeline host logic (RustGS/src/training/data/frame_loader.rs and
its tests) and the oracle's target conversion (frame_targets.rs and its
tests): no GPU needed."""
import numpy as np
import pytest

from oracle import oracle as O
from rustscan_b200 import frames as F


def _flat(frame_count, batch, seed):
    return [i for b in F.DeterministicFrameBatchIter(frame_count, batch, seed) for i in b]


def test_batch_iterator_repeats_for_same_seed():
    a, b = _flat(6, 2, 7), _flat(6, 2, 7)
    assert a == b
    assert sorted(a) == [0, 1, 2, 3, 4, 5]


def test_batch_iterator_changes_order_with_seed():
    assert _flat(6, 2, 7) != _flat(6, 2, 11)


def test_ordered_frame_indices_matches_batch_iterator():
    assert F.ordered_frame_indices(8, 3, 19) == _flat(8, 3, 19)


def test_batch_iterator_shapes():
    assert _flat(5, 2, 0) == [0, 1, 2, 3, 4]  # seed 0 keeps the dataset order
    assert [len(b) for b in F.DeterministicFrameBatchIter(5, 2, 3)] == [2, 2, 1]
    assert [len(b) for b in F.DeterministicFrameBatchIter(3, 0, 3)] == [1, 1, 1]  # batch size at least 1


def test_splitmix64_first_outputs():
    # SplitMix64 seeded with 0: the first outputs of the published generator.
    g = F.SplitMix64(0)
    assert [g.next_u64() for _ in range(3)] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]


def test_worker_count_respects_prefetch_ahead_and_frame_count():
    assert F.frame_loader_worker_count(1, F.FrameLoaderOptions(8, 8)) == 1
    assert F.frame_loader_worker_count(3, F.FrameLoaderOptions(8, 2)) == 2
    assert F.frame_loader_worker_count(16, F.FrameLoaderOptions(8, 8), parallelism=3) == 3


def _decode(i):
    img = np.zeros((2, 3, 3), np.uint8)
    img[0, 0, 0] = i + 1
    return img


def test_prefetch_cache_stays_within_capacity_and_evicts_old_frames():
    loader = F.PrefetchFrameLoader(_decode, 4, F.FrameLoaderOptions(cache_capacity=2, prefetch_ahead=3))
    try:
        order = F.DeterministicFrameBatchIter(4, 1, 3).order()
        loader.prefetch_order_window(order, 0)
        first, second, third = order[0], order[1], order[2]
        f0 = loader.get(first)
        assert int(f0.rgb[0, 0, 0]) == first + 1
        assert (f0.height, f0.width) == (2, 3)
        loader.prefetch_order_window(order, 1)
        loader.get(second)
        loader.get(third)
        assert loader.cache_len() <= 2
        assert not loader.is_cached(first)
        assert loader.is_cached(second) or loader.is_cached(third)
    finally:
        loader.close()


def test_loader_errors():
    with pytest.raises(F.FrameLoadError, match="does not contain any poses"):
        F.PrefetchFrameLoader(_decode, 0)

    def bad(i):
        if i == 1:
            raise OSError("unreadable image")
        return _decode(i)

    loader = F.PrefetchFrameLoader(bad, 3, F.FrameLoaderOptions(cache_capacity=4, prefetch_ahead=1))
    try:
        with pytest.raises(F.FrameLoadError, match="outside the dataset bounds"):
            loader.get(3)
        assert int(loader.get(0).rgb[0, 0, 0]) == 1
        with pytest.raises(OSError, match="unreadable"):
            loader.get(1)
        with pytest.raises(F.FrameLoadError, match="shape"):
            F.DecodedFrame(np.zeros((2, 2), np.uint8))
    finally:
        loader.close()


def test_oracle_frame_to_target_known_answers():
    # frame_targets/tests.rs: identity dimensions map each byte to b / 255.
    r = O.frame_to_target(np.array([0, 64, 255, 255, 128, 0], np.uint8), 2, 1, 2, 1).reshape(-1)
    assert r.shape == (6,)
    assert abs(r[0] - 0.0) < 1e-6 and abs(r[1] - 64.0 / 255.0) < 1e-6 and abs(r[2] - 1.0) < 1e-6
    # A 2x2 frame to 1x1 averages its four pixels per channel.
    src = np.arange(12, dtype=np.uint8)
    r = O.frame_to_target(src, 2, 2, 1, 1).reshape(-1)
    np.testing.assert_allclose(r, [(0 + 3 + 6 + 9) / 4 / 255, (1 + 4 + 7 + 10) / 4 / 255, (2 + 5 + 8 + 11) / 4 / 255],
                               rtol=1e-6)
    # Upscaling repeats source pixels (every box holds one source pixel).
    r = O.frame_to_target(np.array([10, 20, 30, 40, 50, 60], np.uint8), 2, 1, 4, 1).reshape(4, 3)
    np.testing.assert_array_equal(r[0], r[1])
    np.testing.assert_array_equal(r[2], r[3])
    with pytest.raises(ValueError):
        O.frame_to_target(np.zeros(5, np.uint8), 2, 1, 2, 1)
