"""Uneven multi-view batches in one launch and the autotuner (the uneven
batch configuration, config 5, restated at a size the CPU oracle finishes
quickly: 30k Gaussians, 12 views of four resolutions at camera distances
U[1.5, 8], so visible counts differ about threefold and image sizes 27-fold
between views).

Every view of the batch is bit-exact against the oracle's single-view
forward; the batched backward equals the sum of the per-view oracle
adjoints; every tile shape and raster batch size gives the same bit-exact
forward; the autotuner returns a runnable configuration whose forward is
again bit-exact; the persistent cost-ordered raster schedule and the
one-CTA-per-tile grid give the same forward bit for bit, gradients within
the parity bar, and bitwise equal gradients in deterministic mode."""
import numpy as np
import pytest

from _parity import assert_forward_parity, assert_grad_parity, oracle_forward, run_gpu_forward
from rustscan_b200 import scenes as S

pytestmark = pytest.mark.gpu

RES = ((80, 60), (160, 120), (320, 240), (480, 270))


def _scene():
    return S.config5(n=30_000, views=12, resolutions=RES)


def _dev(scene):
    from rustscan_b200 import host_splats_to_device

    return host_splats_to_device(scene)


@pytest.mark.parametrize("schedule", ["persistent", "grid"])
def test_uneven_batch_forward_and_backward(gsr_ctx_factory, schedule):
    import torch

    sc = _scene()
    nv = len(sc.cameras)
    counts = []
    ctx = gsr_ctx_factory(max_splats=sc.n, max_views=nv, max_pixels=max(w * h for w, h in RES), schedule=schedule)
    splats = _dev(sc)
    _, g = run_gpu_forward(ctx, splats, sc.cameras)
    ups = [S.upstream_grad(c.height, c.width, seed=v) for v, c in enumerate(sc.cameras)]
    grads = ctx.render_backward(splats, torch.as_tensor(np.concatenate([u.reshape(-1) for u in ups]), device="cuda"))
    torch.cuda.synchronize()
    keys = ("v_transforms", "v_sh", "v_raw_opacity")
    r32 = {k: 0.0 for k in keys}
    r64 = {k: 0.0 for k in keys}
    for v, cam in enumerate(sc.cameras):
        o = oracle_forward(sc, cam)
        assert_forward_parity(g[v], o)
        counts.append(o.num_visible)
        b32 = o.backward(ups[v], mode=0)
        b64 = oracle_forward(sc, cam, f64=True).backward(ups[v], mode=0)
        for k in keys:
            r32[k] = r32[k] + b32[k]
            r64[k] = r64[k] + b64[k]
    assert max(counts) > 2 * max(1, min(counts)), counts  # genuinely uneven
    for k in keys:
        assert_grad_parity(grads[k].cpu().numpy(), r32[k], r64[k], what=k)


@pytest.mark.parametrize("tile", [(16, 16), (8, 8), (32, 8)])
@pytest.mark.parametrize("batch", [64, 128, 256])
def test_tile_shapes_and_batches_bit_exact(gsr_ctx_factory, tile, batch):
    sc = S.small_scene(n=5000, degree=3, width=112, height=84, seed=120, views=2)
    ctx = gsr_ctx_factory(max_splats=sc.n, max_views=2, max_pixels=112 * 84, tile=tile, batch=batch)
    splats = _dev(sc)
    _, g = run_gpu_forward(ctx, splats, sc.cameras)
    for v, cam in enumerate(sc.cameras):
        assert_forward_parity(g[v], oracle_forward(sc, cam, tile=tile))


def test_autotune_picks_a_runnable_configuration(gsr_ctx_factory):
    from rustscan_b200 import autotune

    sc = _scene()
    nv = len(sc.cameras)
    splats = _dev(sc)
    res = autotune(splats, sc.cameras, reps=2, max_pixels=max(w * h for w, h in RES))
    assert len(res["candidates"]) == 9
    ok = [c for c in res["candidates"] if c["status"] == 0]
    assert ok and all(c["ms_per_view"] > 0 for c in ok)
    assert res["ms_per_view"] == min(c["ms_per_view"] for c in ok)
    ctx = gsr_ctx_factory(max_splats=sc.n, max_views=nv, max_pixels=max(w * h for w, h in RES), tile=res["tile"],
                          batch=res["batch"], max_isects=4 << 20)
    _, g = run_gpu_forward(ctx, splats, sc.cameras)
    for v in (0, nv - 1):
        assert_forward_parity(g[v], oracle_forward(sc, sc.cameras[v], tile=res["tile"]))


@pytest.mark.parametrize("tile", [(16, 16), (8, 8), (32, 8)])
def test_schedules_agree(gsr_ctx_factory, tile):
    """Persistent and grid schedules: identical images and per-pixel state,
    gradients within the parity bar of each other's oracle, and in
    deterministic mode bitwise identical gradients."""
    import torch

    sc = _scene()
    nv = len(sc.cameras)
    pmax = max(w * h for w, h in RES)
    splats = _dev(sc)
    ups = torch.as_tensor(np.concatenate([S.upstream_grad(c.height, c.width, seed=v).reshape(-1)
                                          for v, c in enumerate(sc.cameras)]), device="cuda")
    out = {}
    for det in (False, True):
        for schedule in ("persistent", "grid"):
            ctx = gsr_ctx_factory(max_splats=sc.n, max_views=nv, max_pixels=pmax, tile=tile, schedule=schedule,
                                  deterministic=det)
            _, g = run_gpu_forward(ctx, splats, sc.cameras)
            gr = ctx.render_backward(splats, ups)
            torch.cuda.synchronize()
            out[(det, schedule)] = (g, {k: gr[k].cpu().numpy() for k in ("v_transforms", "v_sh", "v_raw_opacity")})
            ctx.close()
    for det in (False, True):
        ga, gb = out[(det, "persistent")][0], out[(det, "grid")][0]
        for v in range(nv):
            for k in ("image", "tfinal", "last", "ncontrib", "nvisit", "hit_blocks", "isect_vals", "visible"):
                np.testing.assert_array_equal(ga[v][k], gb[v][k], err_msg=f"{k} view {v}")
    for k in ("v_transforms", "v_sh", "v_raw_opacity"):
        np.testing.assert_array_equal(out[(True, "persistent")][1][k], out[(True, "grid")][1][k])
        a, b = out[(False, "persistent")][1][k], out[(False, "grid")][1][k]
        assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b), k


def test_sixty_four_views_in_one_batch(gsr_ctx_factory):
    """The largest batch the context accepts (64 views): every view's
    projection records (visibility masks, compact indices) and forward are
    bit-exact against the oracle, and the batched backward equals the sum of
    the per-view oracle adjoints. 3001 Gaussians leave a partial last
    projection block."""
    import torch

    sc = S.small_scene(n=3001, degree=2, width=48, height=40, seed=164, views=64)
    nv = len(sc.cameras)
    ctx = gsr_ctx_factory(max_splats=sc.n, max_views=nv, max_pixels=48 * 40)
    splats = _dev(sc)
    _, g = run_gpu_forward(ctx, splats, sc.cameras)
    ups = [S.upstream_grad(c.height, c.width, seed=300 + v) for v, c in enumerate(sc.cameras)]
    grads = ctx.render_backward(splats, torch.as_tensor(np.concatenate([u.reshape(-1) for u in ups]), device="cuda"))
    torch.cuda.synchronize()
    keys = ("v_transforms", "v_sh", "v_raw_opacity")
    r32 = {k: 0.0 for k in keys}
    r64 = {k: 0.0 for k in keys}
    for v, cam in enumerate(sc.cameras):
        o = oracle_forward(sc, cam)
        assert_forward_parity(g[v], o)
        b32 = o.backward(ups[v], mode=0)
        b64 = oracle_forward(sc, cam, f64=True).backward(ups[v], mode=0)
        for k in keys:
            r32[k] = r32[k] + b32[k]
            r64[k] = r64[k] + b64[k]
    for k in keys:
        assert_grad_parity(grads[k].cpu().numpy(), r32[k], r64[k], what=k)


def test_one_and_two_pixel_wide_views(gsr_ctx_factory):
    """Views of 1x1, 2x1, 1x40 and 40x1 pixels in one batch (one tile or a
    row or column of tiles each): every view's forward bit-exact, and the
    batched backward equal to the sum of the per-view oracle adjoints."""
    import torch

    base = S.small_scene(n=1500, degree=3, width=64, height=48, seed=170, views=1)
    c = base.cameras[0]
    cams = [S.Camera(c.viewmat, c.fx, c.fy, w * 0.5, h * 0.5, w, h, c.campos) for (w, h) in
            ((1, 1), (2, 1), (1, 40), (40, 1))]
    ctx = gsr_ctx_factory(max_splats=base.n, max_views=len(cams), max_pixels=40)
    splats = _dev(base)
    _, g = run_gpu_forward(ctx, splats, cams)
    ups = [S.upstream_grad(cam.height, cam.width, seed=400 + v) for v, cam in enumerate(cams)]
    grads = ctx.render_backward(splats, torch.as_tensor(np.concatenate([u.reshape(-1) for u in ups]), device="cuda"))
    torch.cuda.synchronize()
    keys = ("v_transforms", "v_sh", "v_raw_opacity")
    r32 = {k: 0.0 for k in keys}
    r64 = {k: 0.0 for k in keys}
    for v, cam in enumerate(cams):
        o = oracle_forward(base, cam)
        assert o.num_visible > 0
        assert_forward_parity(g[v], o)
        b32 = o.backward(ups[v], mode=0)
        b64 = oracle_forward(base, cam, f64=True).backward(ups[v], mode=0)
        for k in keys:
            r32[k] = r32[k] + b32[k]
            r64[k] = r64[k] + b64[k]
    for k in keys:
        assert_grad_parity(grads[k].cpu().numpy(), r32[k], r64[k], what=k)
