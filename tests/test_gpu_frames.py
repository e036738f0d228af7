"""Device conversion of 8-bit frames to training targets
(gsr_frames_to_targets; frame_targets.rs:44-62) bit-exact against the
oracle's restatement, and the frame-fed training step against the step on
targets converted by the oracle."""
import numpy as np
import pytest

from _parity import oracle_forward
from oracle import oracle as O
from rustscan_b200 import scenes as S

pytestmark = pytest.mark.gpu


def _cam(w, h):
    return S.camera_from_rt(np.eye(3), np.zeros(3), 50, 50, w / 2, h / 2, w, h)


@pytest.mark.parametrize("sizes", [
    [((64, 48), (64, 48))],                                   # identity
    [((128, 96), (64, 48)), ((100, 75), (64, 48))],           # downscale, uneven ratio
    [((33, 17), (64, 48)), ((64, 48), (64, 48)), ((7, 300), (20, 30))],  # upscale, identity, mixed
])
def test_frames_to_targets_match_oracle(gsr_ctx_factory, sizes):
    import torch

    rng = np.random.default_rng(len(sizes))
    frames = [rng.integers(0, 256, (sh, sw, 3), dtype=np.uint8) for (sw, sh), _ in sizes]
    cams = [_cam(dw, dh) for _, (dw, dh) in sizes]
    buf = np.concatenate([f.reshape(-1) for f in frames])
    offs = np.concatenate([[0], np.cumsum([f.size for f in frames])[:-1]])
    descs = [(int(o), sw, sh) for o, ((sw, sh), _) in zip(offs, sizes)]
    ctx = gsr_ctx_factory(max_splats=16, max_views=len(sizes), max_pixels=64 * 48)
    out = ctx.frames_to_targets(torch.as_tensor(buf, device="cuda"), descs, cams)
    torch.cuda.synchronize()
    ref = np.concatenate([O.frame_to_target(f, sw, sh, dw, dh).reshape(-1)
                          for f, ((sw, sh), (dw, dh)) in zip(frames, sizes)])
    np.testing.assert_array_equal(out.cpu().numpy(), ref)


def test_frames_to_targets_rejects_bad_input(gsr_ctx_factory):
    import torch

    from rustscan_b200 import GsrError

    ctx = gsr_ctx_factory(max_splats=16)
    buf = torch.zeros(64 * 48 * 3, dtype=torch.uint8, device="cuda")
    with pytest.raises(GsrError) as ei:
        ctx.frames_to_targets(buf, [(0, 0, 48)], [_cam(64, 48)])
    assert ei.value.status == 1
    with pytest.raises(GsrError) as ei:
        ctx.frames_to_targets(buf, [(0, 64, 48)] * 65, [_cam(2, 2)] * 65)
    assert ei.value.status == 1


@pytest.mark.parametrize("prefetch", [True, False])
def test_frame_fed_step_equals_oracle_targets(gsr_ctx_factory, prefetch):
    """Trainer.train_step_frames (bytes copied on a side stream, prefetched
    by the step before or copied by the step itself, converted on the device
    while the forward runs) is bit-identical to train_step on the oracle's
    f32 targets of the same frames, over a sequence that changes frames and
    resizes one view."""
    import torch

    from rustscan_b200 import LearningRates, Trainer, host_splats_to_device

    sc = S.small_scene(n=1500, degree=3, width=64, height=48, seed=95, views=2)
    rng = np.random.default_rng(5)
    src_sizes = [(64, 48), (128, 96)]  # view 1 is box-averaged down to 64x48
    seqs = [[rng.integers(0, 256, (h, w, 3), dtype=np.uint8) for (w, h) in src_sizes] for _ in range(3)]
    order = [0, 1, 1, 2, 0]
    host = [[torch.from_numpy(f).pin_memory() for f in fs] for fs in seqs]
    lrs = LearningRates()
    ctx_a = gsr_ctx_factory(max_splats=sc.n, max_views=2, max_pixels=64 * 48, deterministic=True)
    ctx_b = gsr_ctx_factory(max_splats=sc.n, max_views=2, max_pixels=64 * 48, deterministic=True)
    sa, sb = host_splats_to_device(sc), host_splats_to_device(sc)
    ta = Trainer(ctx_a, sa, lrs, use_graph=True, total_iterations=100)
    tb = Trainer(ctx_b, sb, lrs, use_graph=True, total_iterations=100)
    for it, k in enumerate(order, start=1):
        nxt = host[order[it]] if prefetch and it < len(order) else None
        la = ta.train_step_frames(sc.cameras, host[k], it, next_frames=nxt).clone()
        tgt = np.concatenate([O.frame_to_target(f, w, h, 64, 48).reshape(-1) for f, (w, h) in zip(seqs[k], src_sizes)])
        lb = tb.train_step(sc.cameras, torch.as_tensor(tgt, device="cuda"), it).clone()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(la.cpu().numpy(), lb.cpu().numpy())
    np.testing.assert_array_equal(sa.transforms.cpu().numpy(), sb.transforms.cpu().numpy())
    np.testing.assert_array_equal(sa.sh_coeffs.cpu().numpy(), sb.sh_coeffs.cpu().numpy())
    with pytest.raises(ValueError):
        ta.train_step_frames(sc.cameras, [torch.from_numpy(seqs[0][0])] * 2, 99)
