"""A seeded sweep over the configuration space against the oracle: random
scene sizes, SH degrees, image shapes (ragged against the tiles, down to a
few pixels), tile shapes, raster batches, schedules, deterministic mode,
background colours and view counts. Every configuration: integer outputs
bit-exact and images within 1e-5 for every view, and gradients (summed over
the views) within the parity bar of the FP32 / FP64 oracles."""
import numpy as np
import pytest

from _parity import assert_forward_parity, assert_grad_parity, oracle_forward, run_gpu_forward
from rustscan_b200 import scenes as S

pytestmark = pytest.mark.gpu

TILES = ((16, 16), (8, 8), (32, 8))


def _case(seed):
    rng = np.random.default_rng(1000 + seed)
    n = int(rng.integers(1, 4000))
    degree = int(rng.integers(0, 5))
    views = int(rng.integers(1, 4))
    base = S.small_scene(n=n, degree=degree, width=64, height=48, seed=200 + seed, views=views,
                         logscale_mu=float(rng.uniform(-4.0, -2.0)))
    cams = []
    for cam in base.cameras:
        w, h = int(rng.integers(3, 200)), int(rng.integers(3, 150))
        f = float(rng.uniform(0.5, 1.5)) * w
        cams.append(S.Camera(cam.viewmat, f, f * float(rng.uniform(0.9, 1.1)), w * float(rng.uniform(0.3, 0.7)),
                             h * float(rng.uniform(0.3, 0.7)), w, h, cam.campos))
    opts = dict(tile=TILES[int(rng.integers(0, 3))], batch=int(rng.choice([0, 64, 128, 256])),
                schedule=str(rng.choice(["default", "persistent", "grid"])), deterministic=bool(rng.integers(0, 2)),
                background=tuple(float(x) for x in rng.uniform(0, 1, 3) * rng.integers(0, 2)),
                adjoint=str(rng.choice(["exact", "reference"])))
    return base, cams, opts


@pytest.mark.parametrize("seed", range(24))
def test_configuration_sweep(gsr_ctx_factory, seed):
    import torch

    from rustscan_b200 import host_splats_to_device

    sc, cams, opts = _case(seed)
    pmax = max(c.width * c.height for c in cams)
    ctx = gsr_ctx_factory(max_splats=max(sc.n, 1), max_views=len(cams), max_pixels=pmax, **opts)
    splats = host_splats_to_device(sc)
    _, g = run_gpu_forward(ctx, splats, cams)
    ups = [S.upstream_grad(c.height, c.width, seed=seed * 7 + v) for v, c in enumerate(cams)]
    gr = ctx.render_backward(splats, torch.as_tensor(np.concatenate([u.reshape(-1) for u in ups]), device="cuda"))
    torch.cuda.synchronize()
    keys = ("v_transforms", "v_sh", "v_raw_opacity")
    r32 = {k: 0.0 for k in keys}
    r64 = {k: 0.0 for k in keys}
    mode = 0 if opts["adjoint"] == "exact" else 1
    for v, cam in enumerate(cams):
        o = oracle_forward(sc, cam, tile=opts["tile"], bg=opts["background"])
        assert_forward_parity(g[v], o)
        b32 = o.backward(ups[v], mode=mode)
        b64 = oracle_forward(sc, cam, tile=opts["tile"], bg=opts["background"], f64=True).backward(ups[v], mode=mode)
        for k in keys:
            r32[k] = r32[k] + b32[k]
            r64[k] = r64[k] + b64[k]
    for k in keys:
        assert_grad_parity(gr[k].cpu().numpy(), r32[k], r64[k], what=f"sweep {seed} {opts} {k}")
