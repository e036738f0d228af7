"""Shared helpers of the parity tests: run a scene through the C ABI and
through the CPU oracle, and compare."""
import numpy as np

from oracle import oracle as O


def run_gpu_forward(ctx, splats, cams):
    import torch

    flat, imgs, vis = ctx.render_forward(splats, cams, visible=True)
    torch.cuda.synchronize()
    out = []
    for v, cam in enumerate(cams):
        H, W = cam.height, cam.width
        d = dict(
            counts=ctx.export(v, "counts"),
            gids=ctx.export(v, "gids"),
            tile_counts=ctx.export(v, "tile_counts"),
            depth_order=ctx.export(v, "depth_order"),
            isect_tiles=ctx.export(v, "isect_tiles"),
            isect_vals=ctx.export(v, "isect_vals"),
            tile_ranges=ctx.export(v, "tile_ranges"),
            tfinal=ctx.export(v, "tfinal").reshape(H, W),
            last=ctx.export(v, "last").reshape(H, W),
            ncontrib=ctx.export(v, "ncontrib").reshape(H, W),
            nvisit=ctx.export(v, "nvisit").reshape(H, W),
            image=imgs[v].cpu().numpy(),
            visible=vis[v].cpu().numpy(),
        )
        out.append(d)
    return flat, out


def oracle_forward(scene, cam, tile=(16, 16), cov_blur=0.3, bg=(0.0, 0.0, 0.0), f64=False):
    return O.Forward(scene.transforms, scene.sh, scene.raw_opacity, scene.sh_degree, cam, cov_blur=cov_blur,
                     background=bg, tile=tile, f64=f64)


def assert_forward_parity(g, o, img_atol=1e-5):
    """Bit-exact integer outputs, image within img_atol."""
    V, I = int(g["counts"][0]), int(g["counts"][1])
    assert V == o.num_visible, (V, o.num_visible)
    assert I == o.num_intersections, (I, o.num_intersections)
    np.testing.assert_array_equal(g["gids"], o.gid.astype(np.uint32))
    np.testing.assert_array_equal(g["tile_counts"], o.count)
    np.testing.assert_array_equal(g["depth_order"], o.order.astype(np.uint32))
    np.testing.assert_array_equal(g["isect_tiles"], o.isect_tile)
    np.testing.assert_array_equal(g["isect_vals"], o.isect_c)
    np.testing.assert_array_equal(g["tile_ranges"], o.ranges)
    np.testing.assert_array_equal(g["ncontrib"], o.ncontrib)
    np.testing.assert_array_equal(g["last"], o.last)
    np.testing.assert_array_equal(g["nvisit"], o.nvisit)
    np.testing.assert_array_equal(g["visible"], o.visible)
    np.testing.assert_allclose(g["tfinal"], o.tfinal, rtol=0, atol=img_atol)
    np.testing.assert_allclose(g["image"], o.image, rtol=0, atol=img_atol)


def rel_err(a, b, floor_frac=1e-3):
    """Element-wise |a-b| / max(|b|, floor) with floor = floor_frac * max|b|."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    floor = max(floor_frac * float(np.abs(b).max(initial=0.0)), 1e-30)
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


def assert_grad_close(a, b, rtol=1e-4, floor_frac=1e-3, what=""):
    """Gradient tolerance: relative 1e-4 per element, with an absolute floor
    of floor_frac * max|reference| for elements that cancel to near zero."""
    e = rel_err(a, b, floor_frac)
    worst = float(e.max(initial=0.0))
    assert worst <= rtol, f"{what}: max rel err {worst:.3e} > {rtol} (at {np.unravel_index(int(e.argmax()), e.shape)})"


def assert_grad_parity(g, r32, r64, rtol=1e-4, floor_frac=1e-3, what=""):
    """Gradient parity against the oracle pair (FP32 and FP64 instantiations).

    1. Norm-wise: ||g - r32|| / ||r32|| <= rtol (the relative error of the
       gradient vector, 1e-4).
    2. Element-wise, anchored on the FP64 truth: every element is within
       rtol of r64 (floor: floor_frac * max|r64|), or no further from r64
       than twice the FP32 oracle's own error there. Elements whose value
       cancels in float (where two correct FP32 roundings legitimately differ
       by more than 1e-4) are held to the FP32 oracle's accuracy.
    """
    g = np.asarray(g, np.float64)
    r32 = np.asarray(r32, np.float64)
    r64 = np.asarray(r64, np.float64)
    nrm = float(np.linalg.norm(r32))
    if nrm > 0:
        ne = float(np.linalg.norm(g - r32)) / nrm
        assert ne <= rtol, f"{what}: norm-wise rel err {ne:.3e} > {rtol}"
    floor = max(floor_frac * float(np.abs(r64).max(initial=0.0)), 1e-30)
    allow = np.maximum(rtol * np.maximum(np.abs(r64), floor), 2.0 * np.abs(r32 - r64))
    bad = np.abs(g - r64) > allow
    if bad.any():
        i = np.unravel_index(int(np.argmax(np.abs(g - r64) / allow)), g.shape)
        raise AssertionError(f"{what}: {int(bad.sum())} elements outside tolerance; worst at {i}: gpu {g[i]:.8g} "
                             f"fp32 oracle {r32[i]:.8g} fp64 oracle {r64[i]:.8g}")
