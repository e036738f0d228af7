"""Frame hand-off host logic and the oracle's target conversion
(RustGS/src/training/data/frame_targets.rs and its tests): no GPU needed."""
import numpy as np
import pytest

from oracle import oracle as O
from rustscan_b200 import frames as F


def test_decoded_frame_shape_and_errors():
    f = F.DecodedFrame(np.arange(18, dtype=np.uint8).reshape(2, 3, 3))
    assert (f.height, f.width) == (2, 3)
    assert int(f.rgb[1, 2, 2]) == 17
    with pytest.raises(F.FrameLoadError, match="shape"):
        F.DecodedFrame(np.zeros((2, 2), np.uint8))


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
