"""Parity at the sizes the numbers are quoted on.

* Config 2 (200,000 Gaussians, SH degree 3, 640x480): GPU backward against
  the oracle in both adjoint modes, and against FP64 central differences
  (step 1e-4) on 256 seeded parameters.
* Config 3 (1,000,000 Gaussians, SH degree 3, 8 views of 1280x720 in one
  launch, the benchmark's workload): every view's forward bit-exact in its
  integer outputs and within 1e-5 in its image against the FP32 oracle, with
  the raster batches the autotuner chooses between (128, 256); the loss
  kernel on view 0; and the gradients of view 0 for the oracle's loss
  gradient as upstream (the other views' upstream zero) against the FP32
  and FP64 oracles.
"""
import numpy as np
import pytest

from _parity import assert_forward_parity, assert_grad_close, assert_grad_parity, oracle_forward, report, \
    run_gpu_forward
from rustscan_b200 import scenes as S

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def _fit(ctx, splats, cams):
    from rustscan_b200 import GsrError

    for _ in range(4):
        try:
            ctx.render_forward(splats, cams, check=True)
            return
        except GsrError as e:
            if e.status != 3:
                raise
            ctx.reserve_isects(int(e.required * 1.15) + 1024)
    raise RuntimeError("could not fit intersection capacity")


def _grads_np(g):
    return {k: (t.cpu().numpy() if t is not None else None) for k, t in g.items()}


@pytest.fixture(scope="module")
def config2():
    return S.config2()


@pytest.mark.parametrize("mode", ["exact", "reference"])
def test_config2_backward_full_size(gsr_ctx_factory, config2, mode):
    import torch

    from rustscan_b200 import host_splats_to_device

    sc = config2
    cam = sc.cameras[0]
    up = S.upstream_grad(cam.height, cam.width)
    ctx = gsr_ctx_factory(max_splats=sc.n, max_pixels=640 * 480, max_isects=8 << 20, adjoint=mode)
    splats = host_splats_to_device(sc)
    _, g = run_gpu_forward(ctx, splats, sc.cameras)
    o = oracle_forward(sc, cam)
    assert_forward_parity(g[0], o)
    gg = _grads_np(ctx.render_backward(splats, torch.as_tensor(up, device="cuda"), stats=True))
    torch.cuda.synchronize()
    m = 0 if mode == "exact" else 1
    ob = o.backward(up, mode=m)
    od = oracle_forward(sc, cam, f64=True).backward(up, mode=m)
    assert_grad_close(ctx.export(0, "splat_grads").reshape(-1, 12), ob["splat_grads"], rtol=1e-3,
                      what="screen-space sums")
    for k in ("v_transforms", "v_sh", "v_raw_opacity"):
        assert_grad_parity(gg[k], ob[k], od[k], what=f"config2 {mode} {k}")
    assert_grad_parity(gg["stats"][0], ob["stats"], od["stats"], what=f"config2 {mode} stats")


def test_config2_gpu_gradient_vs_central_differences(gsr_ctx_factory, config2):
    """The GPU's exact adjoint at 256 seeded parameters against FP64 central
    differences (step 1e-4) of the oracle's render, with the FP32 oracle's
    own gradient as the yardstick (assert_grad_parity with the differences in
    the FP64 role). Parameters whose step flips a blend decision are set
    aside (tests/_fd.py)."""
    import torch

    from _fd import analytic, local_central_differences, sample_params
    from oracle import oracle as O
    from rustscan_b200 import host_splats_to_device

    sc = config2
    cam = sc.cameras[0]
    up = S.upstream_grad(cam.height, cam.width)
    base64 = O.Forward(sc.transforms.astype(np.float64), sc.sh.astype(np.float64),
                       sc.raw_opacity.astype(np.float64), 3, cam, f64=True)
    params = sample_params(base64, 256, seed=2)
    fd, flips, _ = local_central_differences(sc, cam, up.astype(np.float64), params, h=1e-4)
    ctx = gsr_ctx_factory(max_splats=sc.n, max_pixels=640 * 480, max_isects=8 << 20)
    splats = host_splats_to_device(sc)
    ctx.render_forward(splats, sc.cameras)
    gg = _grads_np(ctx.render_backward(splats, torch.as_tensor(up, device="cuda"), stats=False))
    r32 = oracle_forward(sc, cam).backward(up, mode=0)
    smooth = ~flips
    g_s = np.array([analytic(gg, p) for p in params])[smooth]
    r_s = np.array([analytic(r32, p) for p in params])[smooth]
    assert flips.sum() <= 0.15 * len(params)
    assert_grad_parity(g_s, r_s, fd[smooth], rtol=1e-4, what="config2 gpu vs fp64 central differences")


# ---- config 3: the benchmark workload ---------------------------------------------


@pytest.fixture(scope="module")
def config3():
    from oracle import oracle as O

    sc = S.config3()
    gt = S.config3_targets()
    cam = sc.cameras[0]
    target = O.Forward(gt[0], gt[1], gt[2], 3, cam).image[..., :3].copy()
    return sc, target


@pytest.mark.parametrize("batch", [128, 256])
def test_config3_forward_all_views(gsr_ctx_factory, config3, batch):
    """All 8 views of one batched launch against the FP32 oracle, view by view."""
    import torch

    from rustscan_b200 import host_splats_to_device

    sc, _ = config3
    ctx = gsr_ctx_factory(max_splats=sc.n, max_views=8, max_pixels=1280 * 720, max_isects=24 << 20, batch=batch)
    splats = host_splats_to_device(sc)
    _fit(ctx, splats, sc.cameras)
    _, g = run_gpu_forward(ctx, splats, sc.cameras)
    torch.cuda.synchronize()
    views = range(8) if batch == 128 else (0, 5)
    for v in views:
        o = oracle_forward(sc, sc.cameras[v])
        assert o.num_intersections > 1_000_000
        assert_forward_parity(g[v], o)
        report(f"config3 view {v} forward (batch {batch})", visible=o.num_visible, intersections=o.num_intersections,
               image_max_abs=float(np.abs(g[v]["image"] - o.image).max()))
        del o
    ctx.close()


def test_config3_view0_loss_and_gradients(gsr_ctx_factory, config3):
    import torch

    from oracle import oracle as O
    from rustscan_b200 import host_splats_to_device

    sc, target = config3
    cams = sc.cameras
    cam = cams[0]
    H, W = cam.height, cam.width
    ctx = gsr_ctx_factory(max_splats=sc.n, max_views=8, max_pixels=1280 * 720, max_isects=24 << 20, batch=128)
    splats = host_splats_to_device(sc)
    _fit(ctx, splats, cams)
    o = oracle_forward(sc, cam)
    val, vp = O.loss(o.image, target)

    # The loss kernel on the oracle's image of view 0.
    loss, vpg = ctx.loss(torch.as_tensor(np.ascontiguousarray(o.image, np.float32), device="cuda"),
                         torch.as_tensor(target, device="cuda"), [cam])
    torch.cuda.synchronize()
    assert abs(float(loss[0]) - val) <= 1e-5 * abs(val), (float(loss[0]), val)
    vpg = vpg.cpu().numpy()
    np.testing.assert_allclose(vpg, vp, rtol=1e-4, atol=1e-4 * float(np.abs(vp).max()))

    # Gradients of view 0 inside the 8-view launch.
    ctx.render_forward(splats, cams)
    up = np.zeros((8, H, W, 4), np.float32)
    up[0] = vp
    gg = _grads_np(ctx.render_backward(splats, torch.as_tensor(up.reshape(-1), device="cuda"), stats=True))
    torch.cuda.synchronize()
    ob = o.backward(vp, mode=0)
    od = oracle_forward(sc, cam, f64=True).backward(vp.astype(np.float64), mode=0)
    for k in ("v_transforms", "v_sh", "v_raw_opacity"):
        assert_grad_parity(gg[k], ob[k], od[k], what=f"config3 view 0 {k}")
    assert_grad_parity(gg["stats"][0], ob["stats"], od["stats"], what="config3 view 0 stats")
    # The other views' gradient columns (signed and absolute mean-gradient
    # sums) are zero under a zero upstream gradient.
    assert not gg["stats"][1:, :, 0:5].any()


def test_unpacked_slot_layout_above_2_20_gaussians(gsr_ctx_factory):
    """1,100,000 Gaussians and a 1280x720 view: the compact index (21 bits)
    and the tile id (12 bits) no longer pack into 32 bits, so the slot
    layout runs with (tile id, compact index) pairs. Forward bit-exact and
    gradients within the parity bar, against the FP32 oracle."""
    import torch

    from rustscan_b200 import host_splats_to_device

    sc = S.config3(n=1_100_000, views=1)
    cam = sc.cameras[0]
    ctx = gsr_ctx_factory(max_splats=sc.n, max_pixels=1280 * 720, max_isects=24 << 20)
    splats = host_splats_to_device(sc)
    _fit(ctx, splats, [cam])
    _, g = run_gpu_forward(ctx, splats, [cam])
    o = oracle_forward(sc, cam)
    assert_forward_parity(g[0], o)
    np.testing.assert_array_equal(ctx.export(0, "tile_counts"), o.count)
    up = S.upstream_grad(cam.height, cam.width)
    gg = _grads_np(ctx.render_backward(splats, torch.as_tensor(up, device="cuda"), stats=False))
    ob = o.backward(up, mode=0)
    od = oracle_forward(sc, cam, f64=True).backward(up, mode=0)
    for k in ("v_transforms", "v_sh", "v_raw_opacity"):
        assert_grad_parity(gg[k], ob[k], od[k], what=f"1.1M unpacked {k}")


@pytest.mark.parametrize("n, size", [(200_000, (640, 480)), (600_000, (1920, 1080)), (30_000, (320, 240))],
                         ids=["packed-11-tile-bits", "pairs-13-tile-bits", "packed-9-tile-bits"])
def test_slot_sort_at_exact_capacity(gsr_ctx_factory, n, size):
    """The slot layout at an intersection capacity equal to the slots
    written, with an odd number of tile-id bits (the sort's digits do not
    split the tile id evenly): every sort position stays inside its
    segment (the sort reports any that would not, instead of writing it)
    and the forward is bit-exact against the oracle. Packed keys and (tile
    id, compact index) pairs."""
    from rustscan_b200 import GsrError, host_splats_to_device

    w, h = size
    sc = S.config3(n=n, views=1, width=w, height=h, focal=1050.0 * w / 1280.0)
    cam = sc.cameras[0]
    ctx = gsr_ctx_factory(max_splats=sc.n, max_pixels=w * h, max_isects=1 << 16)
    splats = host_splats_to_device(sc)
    with pytest.raises(GsrError) as ei:
        ctx.render_forward(splats, [cam], check=True)
    assert ei.value.status == 3
    ctx.reserve_isects(ei.value.required)
    _, g = run_gpu_forward(ctx, splats, [cam])  # raises on any status, the sort's range check included
    assert_forward_parity(g[0], oracle_forward(sc, cam))


# ---- configs 4 and 5 at their stated sizes ---------------------------------------


def test_config4_full_size_bf16_fp64_conic(gsr_ctx_factory):
    """Config 4 as stated: 3,000,000 Gaussians (5% with one log-scale at -9),
    SH degree 3 in BF16 storage, one 1920x1080 view at fx = fy = 1400, the
    FP64 conic. Against the oracle in FP64-conic mode fed the stored
    (BF16-rounded) SH: integer outputs bit-exact, image within 1e-5,
    gradients within the parity bar."""
    import torch

    from oracle import oracle as O
    from rustscan_b200 import host_splats_to_device

    sc = S.config4()
    cam = sc.cameras[0]
    sh_r = torch.as_tensor(sc.sh).to(torch.bfloat16).to(torch.float32).numpy()
    ctx = gsr_ctx_factory(max_splats=sc.n, max_pixels=1920 * 1080, max_isects=48 << 20, sh_dtype="bf16",
                          fp64_conic=True)
    splats = host_splats_to_device(sc, sh_dtype=torch.bfloat16)
    _fit(ctx, splats, [cam])
    _, g = run_gpu_forward(ctx, splats, [cam])
    o = O.Forward(sc.transforms, sh_r, sc.raw_opacity, 3, cam, fp64_conic=True)
    assert o.num_intersections > 10_000_000
    assert_forward_parity(g[0], o)
    up = S.upstream_grad(cam.height, cam.width)
    gg = _grads_np(ctx.render_backward(splats, torch.as_tensor(up, device="cuda"), stats=False))
    ob = o.backward(up, mode=0)
    od = O.Forward(sc.transforms, sh_r, sc.raw_opacity, 3, cam, f64=True, fp64_conic=True).backward(
        up.astype(np.float64), mode=0)
    for k in ("v_transforms", "v_sh", "v_raw_opacity"):
        assert_grad_parity(gg[k], ob[k], od[k], what=f"config4 {k}")
    ctx.close()


def test_config5_full_size_views_bit_exact(gsr_ctx_factory):
    """Config 5 as stated: 2,000,000 Gaussians, 32 views of mixed resolution
    in one launch per stage, BF16 SH storage. One view of each resolution
    (and the view with the fewest visible Gaussians) against the oracle fed
    the stored SH: integer outputs bit-exact, images within 1e-5."""
    import torch

    from oracle import oracle as O
    from rustscan_b200 import host_splats_to_device

    sc = S.config5()
    cams = sc.cameras
    pmax = max(c.width * c.height for c in cams)
    sh_r = torch.as_tensor(sc.sh).to(torch.bfloat16).to(torch.float32).numpy()
    ctx = gsr_ctx_factory(max_splats=sc.n, max_views=len(cams), max_pixels=pmax, max_isects=24 << 20,
                          sh_dtype="bf16")
    splats = host_splats_to_device(sc, sh_dtype=torch.bfloat16)
    _fit(ctx, splats, cams)
    _, g = run_gpu_forward(ctx, splats, cams)
    picks = {}
    for v, c in enumerate(cams):
        picks.setdefault((c.width, c.height), v)
    picks = sorted(set(picks.values()) | {int(np.argmin([int(d["counts"][0]) for d in g]))})
    for v in picks:
        o = O.Forward(sc.transforms, sh_r, sc.raw_opacity, 3, cams[v])
        assert_forward_parity(g[v], o)
        report(f"config5 view {v} forward ({cams[v].width}x{cams[v].height})", visible=o.num_visible,
               intersections=o.num_intersections)
        del o
    ctx.close()  # large capacities: released now, not at the end of the session


@pytest.mark.parametrize("size, tile", [((2560, 1440), (16, 16)), ((1920, 1080), (8, 8))])
def test_more_tiles_than_emission_histograms_cover(gsr_ctx_factory, size, tile):
    """Views with more than 8,192 tiles (14,400 and 32,400 here): emission
    no longer counts intersections per tile, so the binning runs its
    counting walk, ranked emission, a histogram pass in the sort and the
    ranges kernel. Forward bit-exact and gradients within the parity bar."""
    import torch

    from rustscan_b200 import host_splats_to_device

    w, h = size
    sc = S.config3(n=100_000, views=1, width=w, height=h, focal=1050.0 * w / 1280.0)
    cam = sc.cameras[0]
    ctx = gsr_ctx_factory(max_splats=sc.n, max_pixels=w * h, max_isects=8 << 20, tile=tile)
    splats = host_splats_to_device(sc)
    _fit(ctx, splats, [cam])
    _, g = run_gpu_forward(ctx, splats, [cam])
    o = oracle_forward(sc, cam, tile=tile)
    assert o.tiles_x * o.tiles_y > 8192
    assert_forward_parity(g[0], o)
    up = S.upstream_grad(cam.height, cam.width)
    gg = _grads_np(ctx.render_backward(splats, torch.as_tensor(up, device="cuda"), stats=False))
    ob = o.backward(up, mode=0)
    od = oracle_forward(sc, cam, tile=tile, f64=True).backward(up, mode=0)
    for k in ("v_transforms", "v_sh", "v_raw_opacity"):
        assert_grad_parity(gg[k], ob[k], od[k], what=f"{w}x{h} {tile} {k}")
    ctx.close()


@pytest.mark.parametrize("mode", ["exact", "reference"])
def test_one_warp_tile_backward_modes(gsr_ctx_factory, mode):
    """A 2560x1440 view has 14,400 16x16 tiles, more than four waves of the
    one-warp-per-tile backward (16 CTAs per SM x 148 SMs x 4 = 9,472), so
    the backward runs one warp per tile: both adjoints against the oracle
    (screen-space sums, parameter gradients, statistics), and deterministic
    mode bitwise equal across runs and within the parity bar of the default
    reduction."""
    import torch

    from rustscan_b200 import host_splats_to_device

    w, h = 2560, 1440
    sc = S.config3(n=100_000, views=1, width=w, height=h, focal=1050.0 * w / 1280.0)
    cam = sc.cameras[0]
    up = S.upstream_grad(cam.height, cam.width)
    m = 0 if mode == "exact" else 1
    o = oracle_forward(sc, cam)
    assert o.tiles_x * o.tiles_y >= 4 * 16 * 148
    ob = o.backward(up, mode=m)
    od = oracle_forward(sc, cam, f64=True).backward(up, mode=m)
    splats = host_splats_to_device(sc)
    runs = {}
    for det in (False, True, True):
        ctx = gsr_ctx_factory(max_splats=sc.n, max_pixels=w * h, max_isects=8 << 20, adjoint=mode, deterministic=det)
        _, g = run_gpu_forward(ctx, splats, [cam])
        assert_forward_parity(g[0], o)
        gg = _grads_np(ctx.render_backward(splats, torch.as_tensor(up, device="cuda"), stats=True))
        torch.cuda.synchronize()
        assert_grad_close(ctx.export(0, "splat_grads").reshape(-1, 12), ob["splat_grads"], rtol=1e-3,
                          what=f"{mode} det={det} screen-space sums")
        for k in ("v_transforms", "v_sh", "v_raw_opacity"):
            assert_grad_parity(gg[k], ob[k], od[k], what=f"{mode} det={det} {k}")
        assert_grad_parity(gg["stats"][0], ob["stats"], od["stats"], what=f"{mode} det={det} stats")
        runs.setdefault(det, []).append(gg)
        ctx.close()
    for k in ("v_transforms", "v_sh", "v_raw_opacity", "stats"):
        np.testing.assert_array_equal(runs[True][0][k], runs[True][1][k], err_msg=k)


def test_config5_batched_backward_against_one_view(gsr_ctx_factory):
    """Config 5 as stated (2,000,000 Gaussians, 32 views of mixed resolution,
    BF16 SH storage), backward of the whole batch in one launch per stage
    with an upstream gradient on one 320x240 view and zeros on the other 31:
    the parameter gradients equal that view's oracle adjoint (FP32 oracle fed
    the stored SH, FP64 oracle beside it) within the parity bar."""
    import torch

    from oracle import oracle as O
    from rustscan_b200 import host_splats_to_device

    sc = S.config5()
    cams = sc.cameras
    pmax = max(c.width * c.height for c in cams)
    sh_r = torch.as_tensor(sc.sh).to(torch.bfloat16).to(torch.float32).numpy()
    ctx = gsr_ctx_factory(max_splats=sc.n, max_views=len(cams), max_pixels=pmax, max_isects=24 << 20,
                          sh_dtype="bf16")
    splats = host_splats_to_device(sc, sh_dtype=torch.bfloat16)
    _fit(ctx, splats, cams)
    ctx.render_forward(splats, cams)
    v = next(i for i, c in enumerate(cams) if (c.width, c.height) == (320, 240))
    up_v = S.upstream_grad(cams[v].height, cams[v].width, seed=5)
    ups = [up_v if i == v else np.zeros((c.height, c.width, 4), np.float32) for i, c in enumerate(cams)]
    gg = _grads_np(ctx.render_backward(splats, torch.as_tensor(np.concatenate([u.reshape(-1) for u in ups]),
                                                               device="cuda"), stats=False))
    torch.cuda.synchronize()
    ob = O.Forward(sc.transforms, sh_r, sc.raw_opacity, 3, cams[v]).backward(up_v, mode=0)
    od = O.Forward(sc.transforms.astype(np.float64), sh_r.astype(np.float64), sc.raw_opacity.astype(np.float64), 3,
                   cams[v], f64=True).backward(up_v.astype(np.float64), mode=0)
    for k in ("v_transforms", "v_sh", "v_raw_opacity"):
        assert_grad_parity(gg[k], ob[k], od[k], what=f"config5 batched backward, view {v} {k}")
    ctx.close()
