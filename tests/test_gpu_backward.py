"""Backward parity through the C ABI: per-Gaussian screen-space gradient
sums and parameter gradients against the CPU oracle (relative 1e-4 with an
absolute floor of 1e-3 x the largest reference value for entries that cancel),
in the exact-adjoint and reference-semantics modes; deterministic mode is
bitwise repeatable. Parameter gradients are checked with assert_grad_parity
(norm-wise 1e-4 against the FP32 oracle, at least as accurate as the FP32
oracle against the FP64 one, and an element-wise screen)."""
import numpy as np
import pytest

from _parity import assert_grad_close, assert_grad_parity, oracle_forward, run_gpu_forward
from rustscan_b200 import scenes as S

pytestmark = pytest.mark.gpu


def _dev(scene):
    from rustscan_b200 import host_splats_to_device

    return host_splats_to_device(scene)


def _backward(ctx, splats, cams, grads_np):
    import torch

    v = torch.as_tensor(np.concatenate([g.reshape(-1) for g in grads_np]), device="cuda")
    g = ctx.render_backward(splats, v, stats=True)
    torch.cuda.synchronize()
    out = {k: (t.cpu().numpy() if t is not None else None) for k, t in g.items()}
    out["splat_grads"] = [ctx.export(i, "splat_grads").reshape(-1, 12) for i in range(len(cams))]
    return out


@pytest.mark.parametrize("mode", ["exact", "reference"])
@pytest.mark.parametrize("degree", [0, 3])
def test_backward_parity_small(gsr_ctx_factory, mode, degree):
    sc = S.small_scene(n=2500, degree=degree, width=96, height=72, seed=30 + degree)
    cam = sc.cameras[0]
    up = S.upstream_grad(cam.height, cam.width, seed=degree)
    up[..., 3] = np.random.default_rng(9).standard_normal(up[..., 3].shape).astype(np.float32) * 0.3
    ctx = gsr_ctx_factory(max_splats=sc.n, max_pixels=96 * 72, adjoint=mode)
    splats = _dev(sc)
    run_gpu_forward(ctx, splats, sc.cameras)
    g = _backward(ctx, splats, sc.cameras, [up])
    m = 0 if mode == "exact" else 1
    ob = oracle_forward(sc, cam).backward(up, mode=m)
    od = oracle_forward(sc, cam, f64=True).backward(up, mode=m)
    assert_grad_close(g["splat_grads"][0], ob["splat_grads"], rtol=1e-3, what="screen-space sums")
    for k in ("v_transforms", "v_sh", "v_raw_opacity"):
        assert_grad_parity(g[k], ob[k], od[k], what=k)
    assert_grad_parity(g["stats"][0], ob["stats"], od["stats"], what="stats")


def test_backward_config1(gsr_ctx_factory):
    """Config 1 at full size with its N(0,1) upstream gradient."""
    sc = S.config1()
    cam = sc.cameras[0]
    up = S.upstream_grad(256, 256)
    ctx = gsr_ctx_factory(max_splats=sc.n, max_pixels=256 * 256)
    splats = _dev(sc)
    run_gpu_forward(ctx, splats, sc.cameras)
    g = _backward(ctx, splats, sc.cameras, [up])
    ob = oracle_forward(sc, cam).backward(up, mode=0)
    od = oracle_forward(sc, cam, f64=True).backward(up, mode=0)
    for k in ("v_transforms", "v_sh", "v_raw_opacity"):
        assert_grad_parity(g[k], ob[k], od[k], what=k)


def test_multi_view_backward_sums_views(gsr_ctx_factory):
    sc = S.small_scene(n=2000, degree=2, width=64, height=48, seed=44, views=3)
    ups = [S.upstream_grad(48, 64, seed=i) for i in range(3)]
    ctx = gsr_ctx_factory(max_splats=sc.n, max_views=3, max_pixels=64 * 48)
    splats = _dev(sc)
    run_gpu_forward(ctx, splats, sc.cameras)
    g = _backward(ctx, splats, sc.cameras, ups)
    ref, ref64 = None, None
    keys = ("v_transforms", "v_sh", "v_raw_opacity")
    for v, cam in enumerate(sc.cameras):
        ob = oracle_forward(sc, cam).backward(ups[v], mode=0)
        od = oracle_forward(sc, cam, f64=True).backward(ups[v], mode=0)
        assert_grad_parity(g["stats"][v], ob["stats"], od["stats"], what=f"stats view {v}")
        ref = ob if ref is None else {k: ref[k] + ob[k] for k in keys}
        ref64 = od if ref64 is None else {k: ref64[k] + od[k] for k in keys}
    for k in keys:
        assert_grad_parity(g[k], ref[k], ref64[k], what=k)


def test_deterministic_mode_bitwise(gsr_ctx_factory):
    sc = S.small_scene(n=4000, degree=3, width=128, height=96, seed=55)
    up = S.upstream_grad(96, 128, seed=3)
    ctx = gsr_ctx_factory(max_splats=sc.n, max_pixels=128 * 96, deterministic=True)
    splats = _dev(sc)
    res = []
    for _ in range(3):
        run_gpu_forward(ctx, splats, sc.cameras)
        res.append(_backward(ctx, splats, sc.cameras, [up]))
    for k in ("v_transforms", "v_sh", "v_raw_opacity", "stats"):
        np.testing.assert_array_equal(res[0][k], res[1][k])
        np.testing.assert_array_equal(res[0][k], res[2][k])
    ob = oracle_forward(sc, sc.cameras[0]).backward(up, mode=0)
    od = oracle_forward(sc, sc.cameras[0], f64=True).backward(up, mode=0)
    assert_grad_parity(res[0]["v_transforms"], ob["v_transforms"], od["v_transforms"], what="v_transforms (det)")


def test_single_splat_backward_known_answer(gsr_ctx_factory):
    """backward/rasterize_bwd/tests.rs:6-54 restated: one Gaussian in one 16x16
    tile with unit upstream gradients gives non-zero gradients, absolute screen
    statistics at least the signed ones, and positive coverage."""
    # A Gaussian that projects to (8.5, 8.5) with a unit-ish conic, opacity 0.9.
    cam = S.camera_from_rt(np.eye(3), np.array([0.0, 0.0, 2.0]), 16, 16, 8.5, 8.5, 16, 16)
    tr = np.array([[0.0, 0.0, 0.0, 1, 0, 0, 0, np.log(0.12), np.log(0.12), np.log(0.12)]], np.float32)
    sh = ((np.array([1.0, 1.0, 1.0]) - 0.5) / S.SH_C0).reshape(1, 1, 3).astype(np.float32)
    op = np.array([np.log(0.9 / 0.1)], np.float32)
    sc = S.Scene(tr, sh, op, 0, [cam])
    ctx = gsr_ctx_factory(max_splats=1, max_pixels=256)
    splats = _dev(sc)
    run_gpu_forward(ctx, splats, [cam])
    up = np.ones((16, 16, 4), np.float32)
    g = _backward(ctx, splats, [cam], [up])
    s = g["splat_grads"][0][0]
    assert np.abs(s[:9]).mean() > 1e-6
    assert abs(s[9]) + abs(s[10]) >= abs(s[0]) + abs(s[1])
    assert s[11] > 0
    ob = oracle_forward(sc, cam).backward(up, mode=0)
    assert_grad_close(g["splat_grads"][0], ob["splat_grads"], rtol=1e-3, what="single splat")


def test_backward_edge_cases(gsr_ctx_factory):
    """The forward's edge scenes through the backward: no Gaussian at all,
    only culled ones (behind the camera, zero quaternion, off screen,
    transparent), one covering the whole image, a single small one and all
    of them together; parameter gradients and statistics against the oracle
    (rows of culled Gaussians zero)."""
    cam = S.camera_from_rt(np.eye(3), np.array([0.0, 0.0, 3.0]), 64, 64, 32, 32, 64, 64)
    rows = []

    def g(pos, ls, q=(1, 0, 0, 0), op=2.0, rgb=(0.9, 0.2, 0.1)):
        tr = np.zeros(10, np.float32)
        tr[0:3] = pos
        tr[3:7] = q
        tr[7:10] = ls
        rows.append((tr, ((np.asarray(rgb) - 0.5) / S.SH_C0).reshape(1, 3), op))

    g((0, 0, -5), (-2, -2, -2))            # behind the camera
    g((0, 0, 0), (0.5, 0.5, 0.5))          # covers the image
    g((0.1, 0.1, 0.5), (-3, -3, -3), q=(0, 0, 0, 0))  # zero quaternion: culled
    g((0.3, -0.2, 0.2), (-3, -2.5, -4))
    g((5, 5, 0), (-3, -3, -3))             # off screen
    g((0.0, 0.0, 0.0), (-3, -3, -3), op=-8.0)  # transparent: culled
    tr = np.stack([r[0] for r in rows])
    sh = np.stack([r[1] for r in rows]).astype(np.float32)
    op = np.asarray([r[2] for r in rows], np.float32)
    up = S.upstream_grad(64, 64, seed=41)
    for sel in ([], [0, 2, 4, 5], [1], [3], [0, 1, 2, 3, 4, 5]):
        sc = S.Scene(tr[sel].reshape(-1, 10), sh[sel].reshape(-1, 1, 3), op[sel].reshape(-1), 0, [cam])
        ctx = gsr_ctx_factory(max_splats=8, max_pixels=64 * 64)
        splats = _dev(sc)
        run_gpu_forward(ctx, splats, [cam])
        gg = _backward(ctx, splats, [cam], [up])
        if not sel:
            assert gg["v_transforms"].shape == (0, 10) and gg["v_raw_opacity"].shape == (0,)
            continue
        ob = oracle_forward(sc, cam).backward(up, mode=0)
        od = oracle_forward(sc, cam, f64=True).backward(up, mode=0)
        for k in ("v_transforms", "v_sh", "v_raw_opacity"):
            assert_grad_parity(gg[k], ob[k], od[k], what=f"{sel} {k}")
        assert_grad_parity(gg["stats"][0], ob["stats"], od["stats"], what=f"{sel} stats")
