"""Shared helpers of the parity tests: run a scene through the C ABI and
through the CPU oracle, and compare.

With GSR_PARITY_REPORT set to a file path, every gradient comparison
appends one JSON line to it (test id, quantity, norm-wise relative error
against the FP32 and FP64 oracles, the FP32 oracle's own error, and the
per-element 50th/99th-percentile and maximum relative errors against FP64),
so a run leaves the measured errors beside its pass/fail verdicts."""
import json
import os

import numpy as np

from oracle import oracle as O


def report(what, **metrics):
    """Append one measurement to $GSR_PARITY_REPORT (no-op when unset)."""
    path = os.environ.get("GSR_PARITY_REPORT")
    if not path:
        return
    rec = {"test": os.environ.get("PYTEST_CURRENT_TEST", "").split(" ")[0], "what": what}
    rec.update({k: (float(v) if isinstance(v, (np.floating, float)) else v) for k, v in metrics.items()})
    with open(path, "a") as fh:
        fh.write(json.dumps(rec) + "\n")


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
            hit_blocks=ctx.export(v, "hit_blocks"),
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
    if "hit_blocks" in g:
        # Per-entry 8x8 blocks that took the Gaussian, defined up to each
        # tile's largest last-contributor index.
        H, W = o.last.shape
        tw, th = o.tile
        tiles_x = (W + tw - 1) // tw
        ys, xs = np.mgrid[0:H, 0:W]
        tile_of_pix = (ys // th) * tiles_x + (xs // tw)
        tile_max = np.zeros(o.tiles_x * o.tiles_y, np.int64)
        np.maximum.at(tile_max, tile_of_pix.reshape(-1), o.last.reshape(-1).astype(np.int64))
        defined = np.arange(I) < tile_max[o.isect_tile]
        ref = o.hit_blocks()
        assert ref.max(initial=0) < 256
        np.testing.assert_array_equal(g["hit_blocks"][defined], ref[defined].astype(np.uint8))
        assert not ref[~defined].any()
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

    1. Norm-wise, the stated tolerance: ||g - r32|| / ||r32|| <= rtol (1e-4,
       the relative error of the gradient vector), and against the FP64
       truth g is no less accurate than the FP32 oracle, up to rtol:
       ||g - r64|| <= ||r32 - r64|| + rtol ||r64||.
    2. On average as accurate as the FP32 oracle: mean |g - r64| <=
       2 mean |r32 - r64| plus 4 FP32 units in the last place of the average
       element (4 * 2^-23 * mean |r64|). The slack is far below the
       summation error of a scene's gradient vector, but a vector of a few
       elements (one Gaussian) otherwise compares two roundings of the same
       few sums, where either order can win by an ulp.
    3. Element-wise screen for localised errors: every element within
       10 rtol of r64 (floor floor_frac * max|r64|), or no further from r64
       than 4x the FP32 oracle's own error there. A per-element 1e-4 bound
       is not a sound requirement for sums of thousands of signed float
       terms: two correct FP32 summation orders differ by several times the
       oracle's error on elements that cancel, and those are screened here
       relative to the oracle's own error instead.
    """
    g = np.asarray(g, np.float64)
    r32 = np.asarray(r32, np.float64)
    r64 = np.asarray(r64, np.float64)
    if g.size:
        e_el = rel_err(g, r64, floor_frac)
        e_or = rel_err(r32, r64, floor_frac)
        n64 = max(float(np.linalg.norm(r64)), 1e-300)
        report(what, n=int(g.size),
               norm_rel_vs_fp32=float(np.linalg.norm(g - r32)) / max(float(np.linalg.norm(r32)), 1e-300),
               norm_rel_vs_fp64=float(np.linalg.norm(g - r64)) / n64,
               oracle_fp32_norm_rel_vs_fp64=float(np.linalg.norm(r32 - r64)) / n64,
               elem_rel_vs_fp64_p50=float(np.quantile(e_el, 0.5)), elem_rel_vs_fp64_p99=float(np.quantile(e_el, 0.99)),
               elem_rel_vs_fp64_max=float(e_el.max()), oracle_fp32_elem_rel_p99=float(np.quantile(e_or, 0.99)))
    nrm = float(np.linalg.norm(r32))
    if nrm > 0:
        ne = float(np.linalg.norm(g - r32)) / nrm
        assert ne <= rtol, f"{what}: norm-wise rel err {ne:.3e} > {rtol}"
        e64 = float(np.linalg.norm(g - r64))
        o64 = float(np.linalg.norm(r32 - r64))
        assert e64 <= o64 + rtol * float(np.linalg.norm(r64)), f"{what}: error vs FP64 {e64:.3e} (oracle {o64:.3e})"
    if g.size:
        tiny = 4.0 * 2.0 ** -23 * float(np.abs(r64).mean()) + 1e-30
        mg, mo = float(np.abs(g - r64).mean()), float(np.abs(r32 - r64).mean())
        assert mg <= 2.0 * mo + tiny, f"{what}: mean error vs FP64 {mg:.3e} > 2x the FP32 oracle's {mo:.3e}"
    floor = max(floor_frac * float(np.abs(r64).max(initial=0.0)), 1e-30)
    allow = np.maximum(10.0 * rtol * np.maximum(np.abs(r64), floor), 4.0 * np.abs(r32 - r64))
    bad = np.abs(g - r64) > allow
    if bad.any():
        i = np.unravel_index(int(np.argmax(np.abs(g - r64) / allow)), g.shape)
        raise AssertionError(f"{what}: {int(bad.sum())} elements outside tolerance; worst at {i}: gpu {g[i]:.8g} "
                             f"fp32 oracle {r32[i]:.8g} fp64 oracle {r64[i]:.8g}")
