"""Host-side trainer logic without a GPU: the learning-rate schedule of
WgpuTrainer::lr_at (RustGS/src/training/engine/trainer.rs:179-191), computed
in f32 with the C library's logf/expf as the reference computes it."""
import math

import numpy as np

from rustscan_b200 import LearningRates, lr_at


def _ulps(a, b):
    a, b = np.float32(a), np.float32(b)
    return abs(int(a.view(np.int32)) - int(b.view(np.int32)))


def test_lr_schedule_endpoints_and_constants():
    assert lr_at(1.6e-4, 1.6e-6, 0, 30000) == float(np.float32(1.6e-4))
    assert _ulps(lr_at(1.6e-4, 1.6e-6, 30000, 30000), 1.6e-6) <= 4
    assert lr_at(1.6e-4, 1.6e-6, 60000, 30000) == lr_at(1.6e-4, 1.6e-6, 30000, 30000)  # clamped at the end
    assert lr_at(5e-3, 0.0, 1234, 30000) == float(np.float32(5e-3))  # final 0: constant
    assert lr_at(5e-3, 6e-3, 1234, 30000) == float(np.float32(5e-3))  # final >= initial: constant
    assert lr_at(5e-3, 1e-4, 1234, 0) == float(np.float32(5e-3))  # no iterations: constant
    # lr_decay_iterations replaces the horizon.
    assert lr_at(1.6e-4, 1.6e-6, 500, 30000, decay_iterations=1000) == lr_at(1.6e-4, 1.6e-6, 15000, 30000)


def test_lr_schedule_is_f32_and_close_to_exact():
    for it in (1, 7, 999, 12345, 29999):
        v = lr_at(1.6e-4, 1.6e-6, it, 30000)
        assert float(np.float32(v)) == v
        exact = 1.6e-4 * math.exp(math.log(1.6e-6 / 1.6e-4) * it / 30000)
        assert abs(v - exact) <= 8 * np.spacing(np.float32(exact)), (it, v, exact)


def test_learning_rates_groups():
    lr = LearningRates(scale_final=5e-5).at(15000, 30000)
    assert lr.position < 1.6e-4 and lr.scale < 5e-3
    assert lr.rotation == np.float32(1e-3) and lr.color == np.float32(2.5e-3) and lr.opacity == np.float32(0.05)
