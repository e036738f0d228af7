"""Forward parity through the C ABI against the CPU oracle: visible set, tile
counts, depth order, sorted intersection keys and values, tile ranges and
per-pixel contributor counts bit-exact; images within 1e-5 absolute."""
import numpy as np
import pytest

from _parity import assert_forward_parity, oracle_forward, run_gpu_forward
from rustscan_b200 import scenes as S

pytestmark = pytest.mark.gpu


def _dev(scene, sh_dtype="f32"):
    import torch

    from rustscan_b200 import host_splats_to_device

    return host_splats_to_device(scene, sh_dtype=torch.bfloat16 if sh_dtype == "bf16" else torch.float32)


def test_config1_full_size(gsr_ctx_factory):
    """Plain FP32 single view at the full config-1 size (16,384 Gaussians, 256x256)."""
    sc = S.config1()
    ctx = gsr_ctx_factory(max_splats=sc.n, max_pixels=256 * 256)
    _, g = run_gpu_forward(ctx, _dev(sc), sc.cameras)
    o = oracle_forward(sc, sc.cameras[0])
    assert o.num_intersections > 10_000
    assert_forward_parity(g[0], o)


@pytest.mark.parametrize("tile", [(16, 16), (8, 8), (32, 8)])
@pytest.mark.parametrize("degree", [0, 1, 2, 3, 4])
def test_small_scenes_tiles_degrees(gsr_ctx_factory, tile, degree):
    sc = S.small_scene(n=3000, degree=degree, width=100, height=75, seed=degree + 10 * tile[0], views=1)
    ctx = gsr_ctx_factory(max_splats=sc.n, max_pixels=100 * 75, tile=tile)
    _, g = run_gpu_forward(ctx, _dev(sc), sc.cameras)
    o = oracle_forward(sc, sc.cameras[0], tile=tile)
    assert_forward_parity(g[0], o)


def test_multi_view_uneven(gsr_ctx_factory):
    """Several views of different sizes in one launch match the oracle view by view."""
    base = S.small_scene(n=4000, degree=3, width=64, height=48, seed=3, views=4)
    sizes = [(64, 48), (120, 90), (33, 17), (200, 10)]
    cams = []
    for cam, (w, h) in zip(base.cameras, sizes):
        c = S.Camera(cam.viewmat, cam.fx * w / 64, cam.fy * w / 64, w / 2, h / 2, w, h, cam.campos)
        cams.append(c)
    ctx = gsr_ctx_factory(max_splats=base.n, max_views=4, max_pixels=120 * 90)
    _, g = run_gpu_forward(ctx, _dev(base), cams)
    for v, cam in enumerate(cams):
        assert_forward_parity(g[v], oracle_forward(base, cam))


def test_config2_full_size(gsr_ctx_factory):
    """200k Gaussians, SH degree 3, 640x480 (the adjoint-check scene)."""
    sc = S.config2()
    ctx = gsr_ctx_factory(max_splats=sc.n, max_pixels=640 * 480, max_isects=8 << 20)
    _, g = run_gpu_forward(ctx, _dev(sc), sc.cameras)
    assert_forward_parity(g[0], oracle_forward(sc, sc.cameras[0]))


def test_background_and_alpha(gsr_ctx_factory):
    sc = S.small_scene(n=800, degree=1, width=48, height=40, seed=21)
    bg = (0.25, 0.5, 1.0)
    ctx = gsr_ctx_factory(max_splats=sc.n, max_pixels=48 * 40, background=bg)
    _, g = run_gpu_forward(ctx, _dev(sc), sc.cameras)
    o = oracle_forward(sc, sc.cameras[0], bg=bg)
    assert_forward_parity(g[0], o)


def test_edge_cases(gsr_ctx_factory):
    """Everything culled, a Gaussian behind the camera, one covering the whole
    image, a zero quaternion and a single Gaussian."""
    cam = S.camera_from_rt(np.eye(3), np.array([0.0, 0.0, 3.0]), 64, 64, 32, 32, 64, 64)
    rows = []
    K = 1

    def g(pos, ls, q=(1, 0, 0, 0), op=2.0, rgb=(0.9, 0.2, 0.1)):
        tr = np.zeros(10, np.float32)
        tr[0:3] = pos
        tr[3:7] = q
        tr[7:10] = ls
        sh = ((np.asarray(rgb) - 0.5) / S.SH_C0).reshape(1, 3)
        rows.append((tr, sh, op))

    g((0, 0, -5), (-2, -2, -2))            # behind the camera
    g((0, 0, 0), (0.5, 0.5, 0.5))          # covers the image
    g((0.1, 0.1, 0.5), (-3, -3, -3), q=(0, 0, 0, 0))  # zero quaternion: culled
    g((0.3, -0.2, 0.2), (-3, -2.5, -4))
    g((5, 5, 0), (-3, -3, -3))             # off screen
    g((0.0, 0.0, 0.0), (-3, -3, -3), op=-8.0)  # transparent: culled
    tr = np.stack([r[0] for r in rows])
    sh = np.stack([r[1] for r in rows]).astype(np.float32).reshape(-1, K, 3)
    op = np.asarray([r[2] for r in rows], np.float32)
    for sel in ([], [0], [1], [2], [3], [0, 1, 2, 3, 4, 5]):
        sc = S.Scene(tr[sel].reshape(-1, 10), sh[sel].reshape(-1, K, 3), op[sel].reshape(-1), 0, [cam])
        ctx = gsr_ctx_factory(max_splats=8, max_pixels=64 * 64)
        _, gg = run_gpu_forward(ctx, _dev(sc), [cam])
        assert_forward_parity(gg[0], oracle_forward(sc, cam))


def test_capacity_overflow_reported_then_fixed(gsr_ctx_factory):
    import torch

    from rustscan_b200 import GsrError

    sc = S.small_scene(n=3000, degree=0, width=96, height=80, seed=4)
    ctx = gsr_ctx_factory(max_splats=sc.n, max_pixels=96 * 80, max_isects=64)
    splats = _dev(sc)
    with pytest.raises(GsrError) as ei:
        ctx.render_forward(splats, sc.cameras, check=True)
    o = oracle_forward(sc, sc.cameras[0])
    # The required capacity counts the binning's intersection slots: with
    # packed keys and a spare tile id, one per tile of each visible
    # Gaussian's tile box (the passing tiles among them are the intersections).
    b = o.box.astype(np.int64)
    slots = int((np.maximum(b[:, 2] - b[:, 0], 0) * np.maximum(b[:, 3] - b[:, 1], 0)).sum())
    assert slots >= o.num_intersections
    assert ei.value.status == 3 and ei.value.required == slots
    ctx.reserve_isects(ei.value.required)
    _, g = run_gpu_forward(ctx, splats, sc.cameras)
    torch.cuda.synchronize()
    assert_forward_parity(g[0], o)


@pytest.mark.slow
def test_config3_size_properties(gsr_ctx_factory):
    """1M Gaussians, 8 views of 1280x720: size-independent properties."""
    import torch

    sc = S.config3()
    ctx = gsr_ctx_factory(max_splats=sc.n, max_views=8, max_pixels=1280 * 720, max_isects=24 << 20)
    _, g = run_gpu_forward(ctx, _dev(sc), sc.cameras)
    torch.cuda.synchronize()
    for d in g:
        V, I = int(d["counts"][0]), int(d["counts"][1])
        assert 0 < V <= sc.n and I == int(d["tile_counts"].sum(dtype=np.uint64))
        t = d["isect_tiles"]
        assert np.all(t[1:] >= t[:-1])
        r = d["tile_ranges"].reshape(-1, 2)
        nz = r[:, 1] > r[:, 0]
        assert int((r[nz, 1] - r[nz, 0]).sum()) == I
        assert np.all(np.diff(d["gids"].astype(np.int64)) > 0)
        img = d["image"]
        assert np.all(np.isfinite(img)) and img[..., 3].min() >= 0 and img[..., 3].max() <= 1
        np.testing.assert_allclose(1.0 - d["tfinal"], img[..., 3], atol=1e-6)
