"""rustscan_b200 — B200-native differentiable Gaussian-splatting rasterizer.

A host-side mirror of RustGS's renderer/trainer API over the C ABI of
``libgsr.so`` (include/gsr.h). PyTorch supplies device memory and streams;
all computation happens in the library's sm_100a kernels.

Reference interfaces mirrored here:
  * ``DeviceSplats``             — RustGS/src/training/engine/splats.rs:13-63
  * ``render_forward``           — RustGS/src/training/forward/mod.rs:156-294
  * ``render_splats_with_visibility`` (autograd op with ``RenderBackward``)
                                 — RustGS/src/training/backward/autodiff.rs:82-251
  * ``prefix_sum_u32`` / ``radix_sort_by_key_u32``
                                 — RustGS/src/training/gpu_primitives/*.rs
  * ``combined_loss``            — RustGS/src/training/engine/loss.rs:112-142
  * ``AdamScaled``               — RustGS/src/training/engine/optimizer.rs:45-163
  * ``Trainer.train_step``       — RustGS/src/training/engine/trainer.rs:253-440
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math

import numpy as np
import torch

from . import _lib
from ._lib import GsrError
from .scenes import Camera, Scene  # noqa: F401  (re-exported)

DEFAULT_RASTER_COV_BLUR = 0.3  # RustGS/src/training/config.rs:7

EXPORT = dict(counts=0, gids=1, depth_order=2, isect_tiles=3, isect_vals=4, tile_ranges=5, tfinal=6, last=7,
              ncontrib=8, splat_grads=9, nvisit=10, tile_counts=11, hit_blocks=12)


def _require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("rustscan_b200 needs a CUDA device (sm_100a); none is available")


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def camera_struct(cam: Camera) -> _lib.gsr_camera:
    c = _lib.gsr_camera()
    for i in range(16):
        c.viewmat[i] = float(cam.viewmat[i])
    c.fx, c.fy, c.cx, c.cy = float(cam.fx), float(cam.fy), float(cam.cx), float(cam.cy)
    c.width, c.height = int(cam.width), int(cam.height)
    for i in range(3):
        c.campos[i] = float(cam.campos[i])
    return c


def camera_array(cams):
    arr = (_lib.gsr_camera * len(cams))()
    for i, cam in enumerate(cams):
        arr[i] = camera_struct(cam)
    return arr


@dataclasses.dataclass
class DeviceSplats:
    """GPU-resident Gaussians in the RustGS packed layout."""

    transforms: torch.Tensor  # [N,10] f32
    sh_coeffs: torch.Tensor  # [N,K,3] f32 or bf16
    raw_opacities: torch.Tensor  # [N] f32
    sh_degree: int

    def num_splats(self) -> int:
        return int(self.transforms.shape[0])

    def struct(self) -> _lib.gsr_splats:
        s = _lib.gsr_splats()
        s.transforms = self.transforms.data_ptr()
        s.sh = self.sh_coeffs.data_ptr()
        s.raw_opacity = self.raw_opacities.data_ptr()
        s.n = self.num_splats()
        s.sh_degree = int(self.sh_degree)
        return s


def host_splats_to_device(scene, device="cuda", sh_dtype=torch.float32) -> DeviceSplats:
    """engine/splats.rs:26-63: upload a host scene."""
    return DeviceSplats(
        torch.as_tensor(np.ascontiguousarray(scene.transforms), device=device),
        torch.as_tensor(np.ascontiguousarray(scene.sh), device=device).to(sh_dtype).contiguous(),
        torch.as_tensor(np.ascontiguousarray(scene.raw_opacity), device=device),
        int(scene.sh_degree),
    )


SCHEDULES = {"default": _lib.GSR_SCHEDULE_DEFAULT, "persistent": _lib.GSR_SCHEDULE_PERSISTENT,
             "grid": _lib.GSR_SCHEDULE_GRID}


def make_config(max_splats, max_views=1, max_pixels=1920 * 1080, max_isects=0, tile=(16, 16), sh_dtype="f32",
                adjoint="exact", deterministic=False, fp64_conic=False, cov_blur=DEFAULT_RASTER_COV_BLUR,
                background=(0.0, 0.0, 0.0), batch=0, schedule="default") -> _lib.gsr_config:
    """The gsr_config of a context (include/gsr.h). schedule: "default",
    "persistent" (cost-ordered work queue) or "grid" (one CTA per tile)."""
    cfg = _lib.gsr_config()
    cfg.cov_blur = float(cov_blur)
    for i in range(3):
        cfg.background[i] = float(background[i])
    cfg.tile_w, cfg.tile_h = int(tile[0]), int(tile[1])
    cfg.batch = int(batch)
    cfg.sh_dtype = _lib.GSR_SH_BF16 if sh_dtype in ("bf16", torch.bfloat16) else _lib.GSR_SH_F32
    cfg.adjoint = _lib.GSR_ADJOINT_REFERENCE if adjoint == "reference" else _lib.GSR_ADJOINT_EXACT
    cfg.deterministic = int(bool(deterministic))
    cfg.fp64_conic = int(bool(fp64_conic))
    cfg.max_splats = int(max_splats)
    cfg.max_views = int(max_views)
    cfg.max_pixels = int(max_pixels)
    cfg.max_isects = int(max_isects)
    cfg.schedule = SCHEDULES[schedule]
    return cfg


def autotune(splats: "DeviceSplats", cameras, reps=3, **config) -> dict:
    """Pick the tile shape and raster batch for this scene and view mix
    (gsr_autotune): times forward + backward of every candidate in a
    temporary context and returns the fastest plus the full table. The
    keyword arguments are those of Context (tile and batch are ignored)."""
    _require_cuda()
    lib = _lib.load()
    config.setdefault("max_splats", splats.num_splats())
    config.setdefault("max_views", len(cameras))
    config.setdefault("max_pixels", max(c.width * c.height for c in cameras))
    cfg = make_config(**config)
    res = _lib.gsr_tune_result()
    sp = splats.struct()
    cams = camera_array(cameras)
    st = lib.gsr_autotune(C.byref(cfg), C.byref(sp), cams, len(cameras), int(reps), C.byref(res), _stream())
    if st != _lib.GSR_OK:
        raise GsrError(st, "gsr_autotune found no candidate that runs")
    table = [dict(tile=(c.tile_w, c.tile_h), batch=c.batch, status=c.status, ms_per_view=c.ms_per_view)
             for c in res.candidates]
    return dict(tile=(res.tile_w, res.tile_h), batch=res.batch, ms_per_view=res.ms_per_view, candidates=table)


class Context:
    """Owns the library context (scratch, saved forward state) for one stream."""

    def __init__(self, max_splats, max_views=1, max_pixels=1920 * 1080, max_isects=0, tile=(16, 16),
                 sh_dtype="f32", adjoint="exact", deterministic=False, fp64_conic=False,
                 cov_blur=DEFAULT_RASTER_COV_BLUR, background=(0.0, 0.0, 0.0), batch=0, schedule="default"):
        _require_cuda()
        self._lib = _lib.load()
        cfg = make_config(max_splats, max_views, max_pixels, max_isects, tile, sh_dtype, adjoint, deterministic,
                          fp64_conic, cov_blur, background, batch, schedule)
        self.cfg = cfg
        self.background = tuple(float(b) for b in background)
        h = C.c_void_p()
        torch.cuda.init()
        st = self._lib.gsr_create(C.byref(cfg), C.byref(h))
        if st != _lib.GSR_OK:
            raise GsrError(st, "gsr_create failed")
        self._h = h
        self._fwd_cams = None

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gsr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != _lib.GSR_OK:
            raise GsrError(st, self._lib.gsr_last_error(self._h).decode())

    # ---- status ------------------------------------------------------------
    def sync_status(self):
        """Synchronise and raise GsrError on capacity overflow or timeout."""
        req = C.c_uint64(0)
        st = self._lib.gsr_sync_status(self._h, _stream(), C.byref(req))
        if st != _lib.GSR_OK:
            err = GsrError(st, self._lib.gsr_last_error(self._h).decode())
            err.required = int(req.value)
            raise err

    def reserve_isects(self, n):
        self._check(self._lib.gsr_reserve_isects(self._h, int(n)))

    # ---- primitives ----------------------------------------------------------
    def prefix_sum_u32(self, x: torch.Tensor) -> torch.Tensor:
        """Inclusive scan (PrefixSumBackend::prefix_sum_u32_primitive)."""
        x = x.contiguous()
        out = torch.empty_like(x)
        if x.numel():
            self._check(self._lib.gsr_prefix_sum_u32(self._h, _ptr(x), _ptr(out), x.numel(), _stream()))
        return out

    def radix_sort_by_key_u32(self, keys: torch.Tensor, vals: torch.Tensor):
        """Stable sort of (key, value) pairs (RadixSortBackend::radix_sort_by_key_u32_primitive)."""
        keys = keys.contiguous()
        vals = vals.contiguous()
        ko = torch.empty_like(keys)
        vo = torch.empty_like(vals)
        if keys.numel():
            self._check(self._lib.gsr_radix_sort_by_key_u32(self._h, _ptr(keys), _ptr(vals), _ptr(ko), _ptr(vo),
                                                            keys.numel(), _stream()))
        return ko, vo

    # ---- render op -------------------------------------------------------------
    def render_forward(self, splats: DeviceSplats, cameras, visible=False, check=True):
        """Render views; returns (images [list of H,W,4 views of one buffer], visible [V,N] or None)."""
        cams = list(cameras)
        total = sum(c.width * c.height for c in cams)
        out = torch.empty(total * 4, dtype=torch.float32, device="cuda")
        vis = torch.empty((len(cams), splats.num_splats()), dtype=torch.float32, device="cuda") if visible else None
        s = splats.struct()
        arr = camera_array(cams)
        self._check(self._lib.gsr_render_forward(self._h, C.byref(s), arr, len(cams), _ptr(out), _ptr(vis),
                                                 _stream()))
        if check:
            self.sync_status()
        self._fwd_cams = cams
        imgs, o = [], 0
        for c in cams:
            n = c.width * c.height * 4
            imgs.append(out[o:o + n].view(c.height, c.width, 4))
            o += n
        return out, imgs, vis

    def render_backward(self, splats: DeviceSplats, v_rgba: torch.Tensor, stats=True):
        """Parameter gradients of the last forward for upstream image gradients."""
        n = splats.num_splats()
        K = (splats.sh_degree + 1) ** 2
        g = dict(
            v_transforms=torch.empty((n, 10), dtype=torch.float32, device="cuda"),
            v_sh=torch.empty((n, K, 3), dtype=torch.float32, device="cuda"),
            v_raw_opacity=torch.empty(n, dtype=torch.float32, device="cuda"),
        )
        nv = len(self._fwd_cams) if self._fwd_cams else 1
        g["stats"] = torch.empty((nv, n, 7), dtype=torch.float32, device="cuda") if stats else None
        gs = _lib.gsr_grads(g["v_transforms"].data_ptr(), g["v_sh"].data_ptr(), g["v_raw_opacity"].data_ptr())
        s = splats.struct()
        v = v_rgba.contiguous()
        self._check(self._lib.gsr_render_backward(self._h, C.byref(s), _ptr(v), C.byref(gs), _ptr(g["stats"]),
                                                  _stream()))
        return g

    def export(self, view, what):
        """Copy internal state of the last forward to the host (numpy)."""
        code = EXPORT[what] if isinstance(what, str) else int(what)
        cnt = np.zeros(2, np.uint32)
        self._check(self._lib.gsr_export(self._h, view, 0, cnt.ctypes.data, 8, _stream()))
        V, I = int(cnt[0]), int(cnt[1])
        cam = self._fwd_cams[view]
        P = cam.width * cam.height
        tx = math.ceil(cam.width / self.cfg.tile_w)
        ty = math.ceil(cam.height / self.cfg.tile_h)
        shapes = {0: (2, np.uint32), 1: (V, np.uint32), 2: (V, np.uint32), 3: (I, np.uint32), 4: (I, np.uint32),
                  5: (2 * tx * ty, np.uint32), 6: (P, np.float32), 7: (P, np.uint32), 8: (P, np.uint32),
                  9: (12 * V, np.float32), 10: (P, np.uint32), 11: (V, np.uint32), 12: (I, np.uint8)}
        if code == 0:
            return cnt
        n, dt = shapes[code]
        out = np.zeros(max(n, 1), dt)
        self._check(self._lib.gsr_export(self._h, view, code, out.ctypes.data, out.nbytes, _stream()))
        return out[:n]

    # ---- loss / optimizer ----------------------------------------------------------
    def loss(self, pred: torch.Tensor, target: torch.Tensor, cameras, l1_weight=0.8, ssim_weight=0.2):
        """combined_loss_with_kernel: per-view loss values and d loss / d pred (RGBA layout)."""
        cams = list(cameras)
        loss = torch.empty(len(cams), dtype=torch.float32, device="cuda")
        vp = torch.empty_like(pred)
        arr = camera_array(cams)
        self._check(self._lib.gsr_loss(self._h, _ptr(pred.contiguous()), _ptr(target.contiguous()), arr, len(cams),
                                       float(l1_weight), float(ssim_weight), _ptr(loss), _ptr(vp), _stream()))
        return loss, vp


def frame_array(descs):
    """(offset, width, height) triples as a gsr_frame array."""
    arr = (_lib.gsr_frame * len(descs))()
    for i, (off, w, h) in enumerate(descs):
        arr[i].offset, arr[i].width, arr[i].height = int(off), int(w), int(h)
    return arr


def _frames_to_targets(ctx, frames: torch.Tensor, descs, cameras, out: torch.Tensor | None = None):
    cams = list(cameras)
    if len(descs) != len(cams):
        raise ValueError("one frame per camera")
    n = sum(c.width * c.height * 3 for c in cams)
    if out is None:
        out = torch.empty(n, dtype=torch.float32, device="cuda")
    if out.numel() < n or not out.is_contiguous() or out.dtype != torch.float32:
        raise ValueError("target buffer too small or not contiguous f32")
    if frames.dtype != torch.uint8 or not frames.is_cuda or not frames.is_contiguous():
        raise ValueError("frames must be a contiguous uint8 device tensor")
    ctx._check(ctx._lib.gsr_frames_to_targets(ctx._h, _ptr(frames), frame_array(descs), camera_array(cams),
                                              len(cams), _ptr(out), _stream()))
    return out


Context.frames_to_targets = _frames_to_targets
Context.frames_to_targets.__doc__ = (
    """Training targets from decoded 8-bit RGB frames on the device
    (gsr_frames_to_targets): frames is a uint8 device buffer, descs the
    (byte offset, width, height) of each view's frame; returns (or fills
    `out`) the packed per-view [H,W,3] f32 targets at the cameras'
    resolutions.""")


def prefix_sum_u32(x: torch.Tensor, ctx: Context | None = None) -> torch.Tensor:
    ctx = ctx or Context(max_splats=max(x.numel(), 1))
    return ctx.prefix_sum_u32(x)


def radix_sort_by_key_u32(keys: torch.Tensor, vals: torch.Tensor, ctx: Context | None = None):
    ctx = ctx or Context(max_splats=max(keys.numel(), 1))
    return ctx.radix_sort_by_key_u32(keys, vals)


def render_forward(ctx: Context, splats: DeviceSplats, camera: Camera, visible=True):
    """forward/mod.rs:156-294 for one view: (image [H,W,4], visible [N])."""
    _, imgs, vis = ctx.render_forward(splats, [camera], visible=visible)
    return imgs[0], (vis[0] if vis is not None else None)


class _RenderFn(torch.autograd.Function):
    """The render op with RenderBackward (backward/autodiff.rs:82-142) as its backward."""

    @staticmethod
    def forward(fctx, ctx, splats, camera, transforms, sh, raw_opacity, stats_leaf):
        img, vis = render_forward(ctx, splats, camera, visible=True)
        fctx.ctx = ctx
        fctx.splats = splats
        fctx.mark_non_differentiable(vis)
        return img.clone(), vis

    @staticmethod
    def backward(fctx, v_img, _v_vis):
        g = fctx.ctx.render_backward(fctx.splats, v_img.contiguous(), stats=True)
        return (None, None, None, g["v_transforms"], g["v_sh"], g["v_raw_opacity"], g["stats"][0])


@dataclasses.dataclass
class RenderSplatsOutput:
    image: torch.Tensor
    visible: torch.Tensor
    screen_grad_stats: torch.Tensor


def render_splats_with_visibility(ctx: Context, splats: DeviceSplats, camera: Camera) -> RenderSplatsOutput:
    """backward/autodiff.rs:240-251: differentiable render; the [N,7] densification
    statistics arrive as the gradient of ``screen_grad_stats`` (autodiff.rs:192-194)."""
    stats_leaf = torch.zeros((splats.num_splats(), 7), device="cuda", requires_grad=True)
    img, vis = _RenderFn.apply(ctx, splats, camera, splats.transforms, splats.sh_coeffs, splats.raw_opacities,
                               stats_leaf)
    return RenderSplatsOutput(img, vis, stats_leaf)


_LIBM = None


def _libm():
    """The C library's single-precision logf/expf, which Rust's f32::ln and
    f32::exp call on Linux."""
    global _LIBM
    if _LIBM is None:
        import ctypes.util

        m = C.CDLL(ctypes.util.find_library("m") or "libm.so.6")
        for fn in (m.logf, m.expf):
            fn.argtypes = [C.c_float]
            fn.restype = C.c_float
        _LIBM = m
    return _LIBM


def lr_at(initial: float, final_value: float, iteration: int, iterations: int, decay_iterations=None) -> float:
    """WgpuTrainer::lr_at (engine/trainer.rs:179-191) in f32: constant when
    final_value <= 0, final_value >= initial or iterations == 0, else
    initial * exp(ln(final / initial) * t) with t = min(iteration, d) / d,
    d = decay_iterations (default: iterations), every operation rounded to
    f32 as the reference computes it."""
    f32 = np.float32
    initial, final_value = f32(initial), f32(final_value)
    if final_value <= 0 or final_value >= initial or iterations == 0:
        return float(initial)
    d = max(int(decay_iterations if decay_iterations is not None else iterations), 1)
    t = f32(min(int(iteration), d)) / f32(d)
    m = _libm()
    ratio = f32(final_value / initial)
    e = f32(m.expf(float(f32(f32(m.logf(float(ratio))) * t))))
    return float(f32(initial * e))


@dataclasses.dataclass
class LearningRates:
    """TrainingOptimizerConfig defaults (RustGS/src/training/config.rs:532-546):
    every group has an initial rate and a final rate (0: constant) with the
    exponential schedule of lr_at; only the position rate decays by default."""

    position: float = 0.00016
    position_final: float = 0.0000016
    rotation: float = 0.001
    rotation_final: float = 0.0
    scale: float = 0.005
    scale_final: float = 0.0
    color: float = 0.0025
    color_final: float = 0.0
    opacity: float = 0.05
    opacity_final: float = 0.0
    decay_iterations: int | None = None
    beta1: float = 0.9
    beta2: float = 0.999
    eps: float = 1e-8

    def at(self, iteration, total):
        """The rates of WgpuTrainer::update_optimizer_lrs (engine/trainer.rs:221-250)
        at `iteration` of `total` training iterations."""
        lr = _lib.gsr_lr()
        lr.position = lr_at(self.position, self.position_final, iteration, total, self.decay_iterations)
        lr.rotation = lr_at(self.rotation, self.rotation_final, iteration, total, self.decay_iterations)
        lr.scale = lr_at(self.scale, self.scale_final, iteration, total, self.decay_iterations)
        lr.color = lr_at(self.color, self.color_final, iteration, total, self.decay_iterations)
        lr.opacity = lr_at(self.opacity, self.opacity_final, iteration, total, self.decay_iterations)
        lr.beta1, lr.beta2, lr.eps = self.beta1, self.beta2, self.eps
        return lr


class AdamScaled:
    """Bias-corrected Adam with per-column learning rates (engine/optimizer.rs:45-163)."""

    def __init__(self, ctx: Context, splats: DeviceSplats, lrs: LearningRates | None = None):
        self.ctx = ctx
        self.lrs = lrs or LearningRates()
        n, K = splats.num_splats(), (splats.sh_degree + 1) ** 2
        z = lambda *s: torch.zeros(s, dtype=torch.float32, device="cuda")  # noqa: E731
        self.m_tr, self.v_tr = z(n, 10), z(n, 10)
        self.m_sh, self.v_sh = z(n, K, 3), z(n, K, 3)
        self.m_op, self.v_op = z(n), z(n)
        self.step = 0

    def state(self):
        return _lib.gsr_adam_state(self.m_tr.data_ptr(), self.v_tr.data_ptr(), self.m_sh.data_ptr(),
                                   self.v_sh.data_ptr(), self.m_op.data_ptr(), self.v_op.data_ptr())

    def reset(self):
        for t in (self.m_tr, self.v_tr, self.m_sh, self.v_sh, self.m_op, self.v_op):
            t.zero_()
        self.step = 0

    def step_device_splats(self, splats: DeviceSplats, grads: dict, lr: _lib.gsr_lr | None = None):
        self.step += 1
        lr = lr or self.lrs.at(0, 0)
        gs = _lib.gsr_grads(grads["v_transforms"].data_ptr(), grads["v_sh"].data_ptr(),
                            grads["v_raw_opacity"].data_ptr())
        st = self.state()
        self.ctx._check(self.ctx._lib.gsr_adam_step(
            self.ctx._h, _ptr(splats.transforms), _ptr(splats.sh_coeffs), _ptr(splats.raw_opacities),
            splats.num_splats(), splats.sh_degree, C.byref(gs), C.byref(st), C.byref(lr), self.step, _stream()))


@dataclasses.dataclass
class TopologyPlan:
    """A topology mutation plan (TopologyMutationPlan, topology/mod.rs:831-870):
    one row per output splat, (source index, kind, sample scalar) with kind one
    of EXISTING, REFINE_EXISTING, REFINE_NEW; pruned splats are the sources no
    row names. refine_decay is (opacity_decay, scale_decay, train_t) or None."""

    EXISTING = _lib.GSR_TOPO_EXISTING
    REFINE_EXISTING = _lib.GSR_TOPO_REFINE_EXISTING
    REFINE_NEW = _lib.GSR_TOPO_REFINE_NEW
    rows: list
    refine_decay: tuple | None = None
    opacity_reset: bool = False
    opacity_reset_cap: float = 0.01  # LITEGS_OPACITY_RESET_CAP (topology/mod.rs:25)


def apply_topology(ctx: Context, splats: DeviceSplats, plan: TopologyPlan, check=True) -> DeviceSplats:
    """apply_mutations (topology/apply.rs:10-27) on the device: returns the
    mutated splat set as new tensors; the input is unchanged. Adam moments and
    densification accumulators are the caller's to reset, as the reference
    does after a topology change."""
    m = len(plan.rows)
    rows = (_lib.gsr_topo_row * max(m, 1))()
    for i, (src, kind, sample) in enumerate(plan.rows):
        rows[i] = _lib.gsr_topo_row(int(src), int(kind), float(sample), 0)
    d_rows = torch.frombuffer(bytearray(rows), dtype=torch.uint8)[: 16 * m].to("cuda") if m else None
    p = _lib.gsr_topo_params()
    if plan.refine_decay is not None:
        p.has_refine_decay = 1
        p.opacity_decay, p.scale_decay, p.train_t = (float(v) for v in plan.refine_decay)
    p.opacity_reset = int(bool(plan.opacity_reset))
    p.opacity_reset_cap = float(plan.opacity_reset_cap)
    K = (splats.sh_degree + 1) ** 2
    out = DeviceSplats(torch.empty((m, 10), dtype=torch.float32, device="cuda"),
                       torch.empty((m, K, 3), dtype=splats.sh_coeffs.dtype, device="cuda"),
                       torch.empty(m, dtype=torch.float32, device="cuda"), splats.sh_degree)
    if m == 0:
        return out
    sp = splats.struct()
    ctx._check(ctx._lib.gsr_topology_apply(ctx._h, C.byref(sp), _ptr(d_rows), m, C.byref(p), _ptr(out.transforms),
                                           _ptr(out.sh_coeffs), _ptr(out.raw_opacities), _stream()))
    if check:
        ctx.sync_status()
    return out


class SplatEvaluationRenderer:
    """training/evaluation/core.rs:343-375 on the GPU: renders splats from a
    camera with the training rasterizer (so evaluation sees what training
    optimises) and returns RGB in [0, 1], [H*W*3], quantised to 1/255 as the
    reference's u8 renderer output is."""

    def __init__(self, render_width: int, render_height: int, raster_cov_blur: float = DEFAULT_RASTER_COV_BLUR,
                 max_splats: int = 1 << 20, background=(0.0, 0.0, 0.0)):
        self.width, self.height = int(render_width), int(render_height)
        self.cov_blur = float(raster_cov_blur)
        self.background = background
        self._max = int(max_splats)
        self._ctx = None

    def _context(self, n):
        if self._ctx is None or n > self._max:
            self._max = max(self._max, n)
            self._ctx = Context(max_splats=self._max, max_pixels=self.width * self.height, cov_blur=self.cov_blur,
                                background=self.background)
        return self._ctx

    def render(self, splats, camera: Camera) -> np.ndarray:
        if not isinstance(splats, DeviceSplats):
            splats = host_splats_to_device(splats)
        if camera.width != self.width or camera.height != self.height:
            raise ValueError("camera size differs from the renderer's")
        ctx = self._context(splats.num_splats())
        flat, _, _ = ctx.render_forward(splats, [camera], check=True)
        rgb = flat.view(self.height, self.width, 4)[..., :3]
        q = torch.round(torch.clamp(rgb, 0.0, 1.0) * 255.0) / 255.0
        return q.reshape(-1).cpu().numpy()


class Trainer:
    """The device part of WgpuTrainer::train_step (engine/trainer.rs:253-440):
    render all views, 0.8 L1 + 0.2 D-SSIM, backward, densification statistics
    (engine/trainer.rs:651-728) and one fused Adam update, optionally replayed
    from a CUDA graph."""

    ACC_NAMES = ("grad_2d", "screen_grad_2d", "abs_grad_2d", "abs_pixel_grad_2d", "pixel_coverage", "camera_depth",
                 "grad_color", "num_observations", "visible_observations")

    def __init__(self, ctx: Context, splats: DeviceSplats, lrs: LearningRates | None = None, total_iterations=30000,
                 l1_weight=0.8, ssim_weight=0.2, use_visible=False, use_graph=True):
        self.ctx = ctx
        self.splats = splats
        self.opt = AdamScaled(ctx, splats, lrs)
        self.total = total_iterations
        self.l1_weight, self.ssim_weight = l1_weight, ssim_weight
        self.use_visible = use_visible
        self.use_graph = use_graph
        self.densify = torch.zeros((9, splats.num_splats()), dtype=torch.float32, device="cuda")
        self.loss = None
        self._cams = None
        self._h2d = None  # host-target pipeline: device targets, staging buffer, copy stream, events
        self._prefetched = None
        self._frames = None  # 8-bit frame pipeline: the same, with a byte staging buffer
        self._frames_prefetched = None

    def train_step(self, cameras, targets: torch.Tensor, iteration: int, targets_ready=None):
        """One training step on the current stream (gsr_train_step). With
        targets_ready (a torch.cuda.Event recorded after the work that writes
        targets), the forward is launched at once and the loss waits on the
        event (gsr_train_step_after). Returns the per-view losses (device)."""
        cams = list(cameras)
        if self.loss is None or self.loss.numel() != len(cams):
            self.loss = torch.zeros(len(cams), dtype=torch.float32, device="cuda")
        self.opt.step += 1
        p = _lib.gsr_train_params()
        # WgpuTrainer::train_step passes iteration.saturating_sub(1) (engine/trainer.rs:362-365).
        p.lr = self.opt.lrs.at(max(iteration - 1, 0), self.total)
        p.step = self.opt.step
        p.l1_weight, p.ssim_weight = self.l1_weight, self.ssim_weight
        p.use_visible = int(self.use_visible)
        if self._cams is not cams:
            self._arr = camera_array(cams)
            self._cams = cams
        st = self.opt.state()
        s = self.splats
        args = (self.ctx._h, _ptr(s.transforms), _ptr(s.sh_coeffs), _ptr(s.raw_opacities), s.num_splats(), s.sh_degree,
                C.byref(st), self._arr, len(cams), _ptr(targets), C.byref(p), _ptr(self.densify), _ptr(self.loss),
                int(self.use_graph))
        if targets_ready is None:
            self.ctx._check(self.ctx._lib.gsr_train_step(*args, _stream()))
        else:
            self.ctx._check(self.ctx._lib.gsr_train_step_after(*args, C.c_void_p(targets_ready.cuda_event), _stream()))
        return self.loss

    def train_step_frames(self, cameras, frames, iteration: int, next_frames=None):
        """One step whose targets are decoded 8-bit RGB frames in pinned host
        memory (frames: one [H,W,3] uint8 tensor per camera, e.g.
        frames.DecodedFrame.rgb).

        On a side stream the bytes (a quarter of the f32 volume) cross to the
        device, unless the previous call was given them as next_frames and
        copied them already, and gsr_frames_to_targets converts them into the
        step's target buffer (resizing frames whose size differs from the
        camera's). Meanwhile the step's forward runs on the current stream;
        its loss waits for the targets (gsr_train_step_after). next_frames,
        if given, start copying while this step runs. Returns the per-view
        losses (device)."""
        cams = list(cameras)
        frames = list(frames)
        if len(frames) != len(cams):
            raise ValueError("one frame per camera")
        for f in frames:
            if f.dtype != torch.uint8 or f.dim() != 3 or f.shape[2] != 3 or not f.is_pinned():
                raise ValueError("frames must be pinned [H,W,3] uint8 tensors")
        if next_frames is not None:
            nxt = list(next_frames)
            if [tuple(f.shape) for f in nxt] != [tuple(f.shape) for f in frames]:
                raise ValueError("next frames must have the shapes of this step's frames")
            for f in nxt:
                if f.dtype != torch.uint8 or not f.is_pinned():
                    raise ValueError("frames must be pinned [H,W,3] uint8 tensors")
        sizes = [f.numel() for f in frames]
        offs = np.concatenate([[0], np.cumsum(sizes)[:-1]]).tolist()
        descs = [(o, f.shape[1], f.shape[0]) for o, f in zip(offs, frames)]
        n_t = sum(c.width * c.height * 3 for c in cams)
        main = torch.cuda.current_stream()
        h = self._frames
        if h is None or h["stage"].numel() < sum(sizes) or h["dev"].numel() != n_t:
            if h is not None:
                main.wait_stream(h["stream"])  # the old buffers are freed in main's order: no reuse under a copy
            h = self._frames = {
                "dev": torch.empty(n_t, dtype=torch.float32, device="cuda"),
                "stage": torch.empty(max(sum(sizes), 1), dtype=torch.uint8, device="cuda"),
                "stream": torch.cuda.Stream(),
                "ready": torch.cuda.Event(),
                "dev_free": torch.cuda.Event(),
            }
            self._frames_prefetched = None
            h["stream"].wait_stream(main)  # the new buffers' allocation is ordered before their use

        def upload(src):
            for f, o, nb in zip(src, offs, sizes):
                h["stage"][o:o + nb].copy_(f.reshape(-1), non_blocking=True)

        cs = h["stream"]
        pre = self._frames_prefetched
        with torch.cuda.stream(cs):
            # Stream order on cs puts the copy after the previous conversion
            # (the last reader of the staging bytes); the conversion waits
            # until the previous step's loss has read the target buffer.
            if not (pre is not None and len(pre) == len(frames) and all(a is b for a, b in zip(pre, frames))):
                upload(frames)
            cs.wait_event(h["dev_free"])
            self.ctx.frames_to_targets(h["stage"], descs, cams, out=h["dev"])
            h["ready"].record(cs)
        loss = self.train_step(cams, h["dev"], iteration, targets_ready=h["ready"])
        h["dev_free"].record(main)
        self._frames_prefetched = None
        if next_frames is not None:
            with torch.cuda.stream(cs):
                upload(nxt)
            self._frames_prefetched = nxt  # held, so the identity check above stays sound
        return loss

    def train_step_host(self, cameras, host_targets: torch.Tensor, iteration: int, next_host_targets=None):
        """One step whose targets live in pinned host memory.

        The targets are copied to the device (or, when the previous call was
        given them as its next_host_targets, taken from the staging buffer
        that call filled on a side stream while its step ran), the step runs
        on the current stream, and next_host_targets, if given, start copying
        into the staging buffer so that the copy overlaps this step. The
        device buffer the step reads stays the same across calls, so a
        captured step graph is replayed, not captured again. Returns the
        per-view losses (device)."""
        if not host_targets.is_pinned():
            raise ValueError("host targets must be in pinned memory")
        main = torch.cuda.current_stream()
        h = self._h2d
        if h is None or h["dev"].shape != host_targets.shape:
            h = self._h2d = {
                "dev": torch.empty(host_targets.shape, dtype=host_targets.dtype, device="cuda"),
                "stage": torch.empty(host_targets.shape, dtype=host_targets.dtype, device="cuda"),
                "stream": torch.cuda.Stream(),
                "ready": torch.cuda.Event(),
                "free": torch.cuda.Event(),
            }
            self._prefetched = None
        if self._prefetched is not None and self._prefetched is host_targets:
            main.wait_event(h["ready"])
            h["dev"].copy_(h["stage"], non_blocking=True)
        else:
            h["dev"].copy_(host_targets, non_blocking=True)
        h["free"].record(main)  # the staging buffer has been read
        loss = self.train_step(cameras, h["dev"], iteration)
        self._prefetched = None
        if next_host_targets is not None:
            if not next_host_targets.is_pinned() or next_host_targets.shape != host_targets.shape:
                raise ValueError("next host targets must be pinned and of the same shape")
            cs = h["stream"]
            cs.wait_event(h["free"])
            with torch.cuda.stream(cs):
                h["stage"].copy_(next_host_targets, non_blocking=True)
            h["ready"].record(cs)
            self._prefetched = next_host_targets
        return loss
