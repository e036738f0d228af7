"""ctypes front end of the CPU oracle (test infrastructure only).

Loads ``oracle/liboracle_gs.so`` (built by ``make -C oracle``) and exposes the
oracle's forward, backward, loss, Adam and densification restatements on
numpy arrays. Only the tests, ``__graft_entry__.smoke()`` and bench.py's CPU
baseline import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_gs.so")
_lib = None

u32p = C.POINTER(C.c_uint32)
i32p = C.POINTER(C.c_int32)
u64p = C.POINTER(C.c_uint64)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_prefix_sum_u32.argtypes = [u32p, u32p, C.c_uint64]
        L.orc_frame_to_target.argtypes = [C.POINTER(C.c_uint8), C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                          f32p]
        L.orc_sort_pairs_u32.argtypes = [u32p, u32p, u32p, u32p, C.c_uint64]
        L.orc_expf.argtypes = [C.c_float]
        L.orc_expf.restype = C.c_float
        L.orc_blend_expf.argtypes = [C.c_float]
        L.orc_blend_expf.restype = C.c_float
        L.orc_logf.argtypes = [C.c_float]
        L.orc_logf.restype = C.c_float
        for suf, fp, ft in (("f32", f32p, C.c_float), ("f64", f64p, C.c_double)):
            f = getattr(L, f"orc_forward_{suf}")
            f.argtypes = [fp, fp, fp, C.c_int, C.c_int, C.c_void_p, ft, fp, C.c_uint32, C.c_uint32, C.c_int]
            f.restype = C.c_void_p
            getattr(L, f"orc_free_{suf}").argtypes = [C.c_void_p]
            getattr(L, f"orc_sizes_{suf}").argtypes = [C.c_void_p, u64p]
            getattr(L, f"orc_visible_{suf}").argtypes = [C.c_void_p, i32p, u32p, fp, fp, u32p]
            getattr(L, f"orc_order_{suf}").argtypes = [C.c_void_p, i32p]
            getattr(L, f"orc_isects_{suf}").argtypes = [C.c_void_p, u32p, u32p, u32p]
            getattr(L, f"orc_hit_blocks_{suf}").argtypes = [C.c_void_p, u32p]
            getattr(L, f"orc_pixels_{suf}").argtypes = [C.c_void_p, fp, fp, u32p, u32p, u32p, fp]
            getattr(L, f"orc_backward_{suf}").argtypes = [C.c_void_p, fp, C.c_int, fp, fp, fp, fp, fp]
            lf = getattr(L, f"orc_loss_{suf}")
            lf.argtypes = [fp, C.c_int, fp, C.c_int, C.c_int, C.c_double, C.c_double, fp]
            lf.restype = C.c_double
        L.orc_adam_f32.argtypes = [f32p, f32p, f32p, f32p, C.c_uint64, f32p, C.c_int, C.c_int] + [C.c_float] * 3
        L.orc_densify_f32.argtypes = [f32p, f32p, f32p, f32p, C.c_int, C.c_int, C.c_int, f32p]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def prefix_sum_u32(x):
    x = np.ascontiguousarray(x, dtype=np.uint32)
    out = np.zeros_like(x)
    lib().orc_prefix_sum_u32(_p(x, u32p), _p(out, u32p), x.size)
    return out


def sort_pairs_u32(keys, vals):
    keys = np.ascontiguousarray(keys, dtype=np.uint32)
    vals = np.ascontiguousarray(vals, dtype=np.uint32)
    ko = np.zeros_like(keys)
    vo = np.zeros_like(vals)
    lib().orc_sort_pairs_u32(_p(keys, u32p), _p(vals, u32p), _p(ko, u32p), _p(vo, u32p), keys.size)
    return ko, vo


def expf(x):
    return lib().orc_expf(float(x))


def logf(x):
    return lib().orc_logf(float(x))


def blend_expf(x):
    return lib().orc_blend_expf(float(x))


class Forward:
    """Oracle forward pass of one view; keeps the inputs alive for the backward."""

    def __init__(self, transforms, sh, raw_opacity, degree, camera, cov_blur=0.3, background=(0.0, 0.0, 0.0),
                 tile=(16, 16), f64=False, fp64_conic=False):
        self.f64 = f64
        dt = np.float64 if f64 else np.float32
        fp = f64p if f64 else f32p
        self.suf = "f64" if f64 else "f32"
        self.dt = dt
        self.transforms = np.ascontiguousarray(transforms, dtype=dt)
        self.sh = np.ascontiguousarray(sh, dtype=dt)
        self.raw_opacity = np.ascontiguousarray(raw_opacity, dtype=dt)
        self.degree = int(degree)
        self.n = int(self.raw_opacity.shape[0])
        self.K = (self.degree + 1) ** 2
        self.camera = camera
        self._cam_rec = camera.as_record()
        self.bg = np.ascontiguousarray(background, dtype=dt)
        self.tile = tile
        L = lib()
        self._h = getattr(L, f"orc_forward_{self.suf}")(
            _p(self.transforms, fp), _p(self.sh, fp), _p(self.raw_opacity, fp), self.n, self.degree,
            self._cam_rec.ctypes.data, (C.c_double if f64 else C.c_float)(cov_blur), _p(self.bg, fp),
            tile[0], tile[1], int(bool(fp64_conic)))
        sizes = np.zeros(4, dtype=np.uint64)
        getattr(L, f"orc_sizes_{self.suf}")(self._h, _p(sizes, u64p))
        self.num_visible, self.num_intersections, self.tiles_x, self.tiles_y = (int(v) for v in sizes)
        V, I = self.num_visible, self.num_intersections
        T = self.tiles_x * self.tiles_y
        H, W = camera.height, camera.width
        self.gid = np.zeros(V, np.int32)
        self.count = np.zeros(V, np.uint32)
        self.depth = np.zeros(V, dt)
        self.rec = np.zeros((V, 10), dt)
        self.box = np.zeros((V, 4), np.uint32)
        getattr(L, f"orc_visible_{self.suf}")(self._h, _p(self.gid, i32p), _p(self.count, u32p),
                                               _p(self.depth, fp), _p(self.rec, fp), _p(self.box, u32p))
        self.order = np.zeros(V, np.int32)
        getattr(L, f"orc_order_{self.suf}")(self._h, _p(self.order, i32p))
        self.isect_tile = np.zeros(I, np.uint32)
        self.isect_c = np.zeros(I, np.uint32)
        self.ranges = np.zeros(2 * T, np.uint32)
        getattr(L, f"orc_isects_{self.suf}")(self._h, _p(self.isect_tile, u32p), _p(self.isect_c, u32p),
                                              _p(self.ranges, u32p))
        self.image = np.zeros((H, W, 4), dt)
        self.tfinal = np.zeros((H, W), dt)
        self.last = np.zeros((H, W), np.uint32)
        self.ncontrib = np.zeros((H, W), np.uint32)
        self.nvisit = np.zeros((H, W), np.uint32)
        self.visible = np.zeros(self.n, dt)
        getattr(L, f"orc_pixels_{self.suf}")(self._h, _p(self.image, fp), _p(self.tfinal, fp), _p(self.last, u32p),
                                              _p(self.ncontrib, u32p), _p(self.nvisit, u32p), _p(self.visible, fp))

    def hit_blocks(self):
        """Per intersection: bits of the tile's 8x8 pixel blocks (x fastest)
        holding a pixel that took the Gaussian."""
        out = np.zeros(max(self.num_intersections, 1), np.uint32)
        getattr(lib(), f"orc_hit_blocks_{self.suf}")(self._h, _p(out, u32p))
        return out[:self.num_intersections]

    def backward(self, v_rgba, mode=0):
        """mode 0: exact adjoint; 1: reference semantics, reverse walk; 2: literal WGSL walk."""
        dt = self.dt
        fp = f64p if self.f64 else f32p
        v = np.ascontiguousarray(v_rgba, dtype=dt)
        out = dict(
            v_transforms=np.zeros((self.n, 10), dt),
            v_sh=np.zeros((self.n, self.K, 3), dt),
            v_raw_opacity=np.zeros(self.n, dt),
            stats=np.zeros((self.n, 7), dt),
            splat_grads=np.zeros((self.num_visible, 12), dt),
        )
        getattr(lib(), f"orc_backward_{self.suf}")(
            self._h, _p(v, fp), int(mode), _p(out["v_transforms"], fp), _p(out["v_sh"], fp),
            _p(out["v_raw_opacity"], fp), _p(out["stats"], fp), _p(out["splat_grads"], fp))
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            try:
                getattr(_lib, f"orc_free_{self.suf}")(h)
            except TypeError:  # interpreter shutdown: ctypes already torn down
                pass
            self._h = None


def frame_to_target(frame_u8, width, height, dst_width, dst_height):
    """resize_rgb_u8_to_f32 (frame_targets.rs:44-62): [height, width, 3] bytes
    to a [dst_height, dst_width, 3] f32 target."""
    src = np.ascontiguousarray(frame_u8, dtype=np.uint8).reshape(-1)
    if src.size != width * height * 3:
        raise ValueError("frame size does not match width x height x 3")
    out = np.zeros((dst_height, dst_width, 3), np.float32)
    lib().orc_frame_to_target(src.ctypes.data_as(C.POINTER(C.c_uint8)), width, height, dst_width, dst_height,
                              _p(out, f32p))
    return out


def loss(pred, target, l1_weight=0.8, ssim_weight=0.2, f64=False):
    """0.8*L1 + 0.2*(1-SSIM) and its gradient; pred is [H,W,3] or [H,W,4]."""
    dt = np.float64 if f64 else np.float32
    fp = f64p if f64 else f32p
    pred = np.ascontiguousarray(pred, dtype=dt)
    target = np.ascontiguousarray(target, dtype=dt)
    H, W, ps = pred.shape
    v = np.zeros_like(pred)
    val = getattr(lib(), f"orc_loss_{'f64' if f64 else 'f32'}")(
        _p(pred, fp), ps, _p(target, fp), H, W, l1_weight, ssim_weight, _p(v, fp))
    return val, v


def adam(param, grad, m, v, lr_cols, step, beta1=0.9, beta2=0.999, eps=1e-8):
    """In-place bias-corrected Adam with a per-column learning rate."""
    lr = np.ascontiguousarray(lr_cols, dtype=np.float32)
    g = np.ascontiguousarray(grad, dtype=np.float32)
    lib().orc_adam_f32(_p(param, f32p), _p(g, f32p), _p(m, f32p), _p(v, f32p), param.size, _p(lr, f32p), lr.size,
                       int(step), float(beta1), float(beta2), float(eps))


def densify(v_transforms, stats, v_sh, visible, acc, use_visible=False):
    n, K = v_sh.shape[0], v_sh.shape[1]
    args = [np.ascontiguousarray(a, dtype=np.float32) for a in (v_transforms, stats, v_sh, visible)]
    lib().orc_densify_f32(*[_p(a, f32p) for a in args], n, K, int(use_visible), _p(acc, f32p))


def ref_cpu_forward(scene, cam, cov_blur=0.3, background=(0.0, 0.0, 0.0)):
    """The reference's shipped single-threaded CPU renderer (tiled_renderer.rs,
    restated in ref_cpu_forward.cpp): returns (colour [H,W,3], depth [H,W]).
    Different semantics from the training path; timed only."""
    L = lib()
    f = L.orc_ref_cpu_forward
    f.restype = None
    tr = np.ascontiguousarray(scene.transforms, np.float32)
    sh = np.ascontiguousarray(scene.sh, np.float32)
    op = np.ascontiguousarray(scene.raw_opacity, np.float32)
    vm = np.ascontiguousarray(cam.viewmat, np.float32)
    cp = np.ascontiguousarray(cam.campos, np.float32)
    bg = np.ascontiguousarray(background, np.float32)
    col = np.zeros((cam.height, cam.width, 3), np.float32)
    dep = np.zeros((cam.height, cam.width), np.float32)
    fp = C.c_void_p
    f(tr.ctypes.data_as(fp), sh.ctypes.data_as(fp), op.ctypes.data_as(fp), C.c_int(op.shape[0]),
      C.c_int(scene.sh_degree), vm.ctypes.data_as(fp), cp.ctypes.data_as(fp), C.c_float(cam.fx), C.c_float(cam.fy),
      C.c_float(cam.cx), C.c_float(cam.cy), C.c_int(cam.width), C.c_int(cam.height), C.c_float(cov_blur),
      bg.ctypes.data_as(fp), col.ctypes.data_as(fp), dep.ctypes.data_as(fp))
    return col, dep


def topology_apply(transforms, sh, raw_opacity, rows, has_decay=False, scale_decay=0.0, opacity_decay=0.0,
                   train_t=0.0, opacity_reset=False, reset_cap=0.01):
    """topology/apply.rs restated: rows is a sequence of (source, kind,
    sample_scalar); returns (transforms [m,10], sh [m,K,3], raw_opacity [m])."""
    L = lib()
    f = L.orc_topology_apply_f32
    f.restype = C.c_int
    tr = np.ascontiguousarray(transforms, np.float32)
    shf = np.ascontiguousarray(sh, np.float32)
    op = np.ascontiguousarray(raw_opacity, np.float32)
    n = op.shape[0]
    m = len(rows)
    rr = np.zeros((m, 3), np.uint32)
    for i, (src, kind, sample) in enumerate(rows):
        rr[i, 0] = src
        rr[i, 1] = kind
        rr[i, 2] = np.float32(sample).view(np.uint32)
    elems = int(np.prod(shf.shape[1:])) if shf.ndim > 1 else 0
    otr = np.zeros((m, 10), np.float32)
    osh = np.zeros((m,) + shf.shape[1:], np.float32)
    oop = np.zeros(m, np.float32)
    fp = C.c_void_p
    st = f(tr.ctypes.data_as(fp), shf.ctypes.data_as(fp), op.ctypes.data_as(fp), C.c_uint32(n), C.c_uint32(elems),
           rr.ctypes.data_as(fp), C.c_uint32(m), C.c_int(int(has_decay)), C.c_float(scale_decay),
           C.c_float(opacity_decay), C.c_float(train_t), C.c_int(int(opacity_reset)), C.c_float(reset_cap),
           otr.ctypes.data_as(fp), osh.ctypes.data_as(fp), oop.ctypes.data_as(fp))
    if st != 0:
        raise ValueError("a plan row names a source out of range")
    return otr, osh, oop

