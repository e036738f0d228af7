"""Central finite differences of a rendered view, evaluated locally.

The scalar is L(theta) = sum(upstream * image) of one view, rendered by the
FP64 oracle. A parameter of Gaussian g changes only g's projection, so the
image can change only in the tiles g touches before or after the step. For
each sampled parameter the difference L(theta + h) - L(theta - h) is
therefore taken over a window of whole tiles (the union of g's tile boxes at
theta - h, theta and theta + h), rendered with the sub-scene of every
Gaussian whose tile box meets that window. Every list of a window tile in the
sub-scene render is the list of the full render (a Gaussian that passes a
tile's test has that tile in its box; relative global-id order, which breaks
depth ties, is kept), so the window pixels are those of a full render and
the difference equals that of two full renders, at a small fraction of the
cost. The camera is never cropped: the Jacobian clamp of helpers.wgsl
(calc_cam_j, helpers.wgsl:138-160) depends on the image width and the
principal point.

A step can flip a discrete decision of the blend (alpha >= 1/255, the
T < 1e-4 termination; rasterize.wgsl:54-88) for some pixel, which the
adjoint does not see and which puts a jump into the difference. Such
parameters are flagged by comparing the per-pixel contributor counts and
last contributors of the two renders over the window.
"""
import numpy as np

from oracle import oracle as O


def _box_of(tr, sh, op, degree, cam, gi, tile):
    """Tile box (x0, y0, x1, y1) of Gaussian gi alone, or None if culled."""
    f = O.Forward(tr[gi:gi + 1], sh[gi:gi + 1], op[gi:gi + 1], degree, cam, tile=tile, f64=True)
    if f.num_visible == 0:
        return None
    return tuple(int(v) for v in f.box[0])


def _union(boxes):
    boxes = [b for b in boxes if b is not None and b[2] > b[0] and b[3] > b[1]]
    if not boxes:
        return None
    return (min(b[0] for b in boxes), min(b[1] for b in boxes), max(b[2] for b in boxes), max(b[3] for b in boxes))


def sample_params(base, n_params, seed):
    """Seeded (kind, gaussian, index) triples over Gaussians that contribute
    to at least one pixel: kind 0 a transforms column (position, quaternion,
    log-scale), 1 an SH coefficient (k, channel), 2 the opacity logit; the
    three kinds equally likely."""
    rng = np.random.default_rng(seed)
    contributing = np.flatnonzero(base.visible > 0)
    K = base.K
    out = []
    for _ in range(n_params):
        gi = int(rng.choice(contributing))
        kind = int(rng.integers(0, 3))
        if kind == 0:
            out.append((0, gi, int(rng.integers(0, 10))))
        elif kind == 1:
            out.append((1, gi, (int(rng.integers(0, K)), int(rng.integers(0, 3)))))
        else:
            out.append((2, gi, 0))
    return out


def analytic(grads, p):
    kind, gi, j = p
    if kind == 0:
        return float(grads["v_transforms"][gi, j])
    if kind == 1:
        return float(grads["v_sh"][gi, j[0], j[1]])
    return float(grads["v_raw_opacity"][gi])


def local_central_differences(scene, cam, upstream, params, h=1e-4, tile=(16, 16)):
    """FP64 central differences (L(+h) - L(-h)) / 2h for each parameter.

    Returns (fd values, flip flags, base forward)."""
    tr = np.asarray(scene.transforms, np.float64)
    sh = np.asarray(scene.sh, np.float64)
    op = np.asarray(scene.raw_opacity, np.float64)
    deg = scene.sh_degree
    up = np.asarray(upstream, np.float64)
    base = O.Forward(tr, sh, op, deg, cam, tile=tile, f64=True)
    n = tr.shape[0]
    gbox = np.zeros((n, 4), np.int64)  # tile box per global id; empty for culled Gaussians
    gbox[base.gid] = base.box.astype(np.int64)
    tw, th = tile
    fds, flips = [], []
    for kind, gi, j in params:
        def perturbed(sign):
            a, b, c = tr, sh, op
            if kind == 0:
                a = tr.copy()
                a[gi, j] += sign * h
            elif kind == 1:
                b = sh.copy()
                b[gi, j[0], j[1]] += sign * h
            else:
                c = op.copy()
                c[gi] += sign * h
            return a, b, c

        plus, minus = perturbed(+1.0), perturbed(-1.0)
        b0 = tuple(gbox[gi]) if gbox[gi, 2] > gbox[gi, 0] else None
        win = _union([b0, _box_of(*plus, deg, cam, gi, tile), _box_of(*minus, deg, cam, gi, tile)])
        if win is None:
            fds.append(0.0)
            flips.append(False)
            continue
        x0, y0, x1, y1 = win
        meets = (gbox[:, 0] < x1) & (gbox[:, 2] > x0) & (gbox[:, 1] < y1) & (gbox[:, 3] > y0)
        meets[gi] = True
        sub = np.flatnonzero(meets)  # ascending: relative global-id order kept
        py0, py1 = y0 * th, min(y1 * th, cam.height)
        px0, px1 = x0 * tw, min(x1 * tw, cam.width)
        res = []
        for a, b, c in (plus, minus):
            f = O.Forward(a[sub], b[sub], c[sub], deg, cam, tile=tile, f64=True)
            img = f.image[py0:py1, px0:px1]
            res.append((float((img * up[py0:py1, px0:px1]).sum()), f.ncontrib[py0:py1, px0:px1].copy(),
                        f.last[py0:py1, px0:px1].copy()))
        fds.append((res[0][0] - res[1][0]) / (2.0 * h))
        # The contributor counts change with g's membership in a pixel's
        # blend; `last` also holds list positions, which shift when g moves
        # in depth order, so only the counts and termination are compared.
        flips.append(not np.array_equal(res[0][1], res[1][1]) or
                     not np.array_equal(res[0][2] > 0, res[1][2] > 0))
    return np.asarray(fds), np.asarray(flips), base
