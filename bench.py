"""Benchmark: forward+backward ms per view of the differentiable Gaussian
rasterizer on the batched training-step workload (1,000,000 Gaussians, SH
degree 3, 8 views of 1280x720 per step, 0.8 L1 + 0.2 D-SSIM, fused Adam and
densification statistics, CUDA-graph replay), next to the plain single-view
path on the same scene.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs its own replica of the workload (the views of
one step do not need another GPU); timings are the max over ranks.
"""
import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+bwd ms/view (1M Gaussians, 1280x720) batched vs plain; grad rel err"
UNIT = "ms/view"
WORKLOAD = "batched training step: 1,000,000 Gaussians, SH degree 3, 8 views of 1280x720 per step"
# ncu smsp__inst_executed.sum of the raster kernels on one 1280x720 view of
# this workload (6,273,269 intersections), per intersection
# (profiles/raster_c3_1view_issue.md).
WARP_INST_PER_ISECT = {"raster_bwd": 153.95e6 / 6273269, "raster_fwd": 134.88e6 / 6273269}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=1_000_000)
    p.add_argument("--views", type=int, default=8)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-bf16", action="store_true", help="skip the BF16-storage batched timing")
    p.add_argument("--no-precision", action="store_true", help="skip the FP64 precision report (CPU baseline leg)")
    p.add_argument("--config", default="c3", choices=["c1", "c3", "c4", "c5"],
                   help="c3 (default): the batched training step the metric is quoted on; c1, c4, c5: the other "
                        "configurations' workloads, one JSON line each")
    p.add_argument("--mode", default="bench", choices=["bench", "profile"],
                   help="profile: warm up, then run exactly one non-graph batched step (for ncu launch lists)")
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        try:
            proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                     "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                    stderr=subprocess.DEVNULL, text=True)
        except Exception:
            return
        while not self._stop.is_set():
            line = proc.stdout.readline()
            if not line:
                break
            self.rows.append([x.strip() for x in line.split(",")])
        proc.terminate()
        try:
            proc.wait(timeout=5)
        except Exception:
            proc.kill()

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        time.sleep(0.3)
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        sm = [float(r[0]) for r in self.rows if r and r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if len(r) > 1 and r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, nm in enumerate(names):
                if len(r) > 4 + i and r[4 + i].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    cuda = torch.cuda.is_available()
    if world > 1:
        import datetime

        import torch.distributed as dist

        if cuda:
            torch.cuda.set_device(local)
        # NCCL between GPUs; gloo where there is none (the host-side checks).
        dist.init_process_group("nccl" if cuda else "gloo", timeout=datetime.timedelta(seconds=300))
    elif cuda:
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(world, x):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def make_context(n, views, sh_dtype="f32", tile=(16, 16), batch=0):
    from rustscan_b200 import Context

    return Context(max_splats=n, max_views=views, max_pixels=1280 * 720, max_isects=24 << 20, sh_dtype=sh_dtype,
                   tile=tile, batch=batch)


def fit_capacity(ctx, splats, cams):
    """Render once; grow the intersection capacity if the scene needs more."""
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


def time_steps(fn, steps, warmup, world):
    import torch

    for i in range(warmup):
        fn(i + 1)
    torch.cuda.synchronize()
    barrier(world)
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    for i in range(steps):
        fn(warmup + i + 1)
    e1.record(st)
    torch.cuda.synchronize()
    barrier(world)
    return max_over_ranks(world, e0.elapsed_time(e1))


def stage_profile(ctx, fn):
    """Per-stage device times (ms) of one call of fn, from CUDA events on the launching stream."""
    import torch

    from rustscan_b200 import _lib

    L = ctx._lib
    L.gsr_profile(ctx._h, 1)
    fn()
    buf = (C.c_float * len(_lib.PROFILE_STAGES))()
    ctx._check(L.gsr_profile_read(ctx._h, buf, len(_lib.PROFILE_STAGES),
                                  C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    L.gsr_profile(ctx._h, 0)
    return {k: float(buf[i]) for i, k in enumerate(_lib.PROFILE_STAGES)}


def _psnr(a, b):
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return float("inf") if mse == 0.0 else 10.0 * np.log10(1.0 / mse)


def _grad_rel(g, r):
    """Norm-wise relative error of the concatenated parameter gradients."""
    keys = ("v_transforms", "v_sh", "v_raw_opacity")
    gv = np.concatenate([np.asarray(g[k], np.float64).reshape(-1) for k in keys])
    rv = np.concatenate([np.asarray(r[k], np.float64).reshape(-1) for k in keys])
    return float(np.linalg.norm(gv - rv) / max(np.linalg.norm(rv), 1e-300))


def cpu_baseline(scene, cams, targets_np, gpu_view=None):
    """CPU baselines on one view of the workload (a bounded sample, ~10-30 s):
    the oracle (C++ restatement of the training path, forward + loss + exact
    backward, OpenMP over all host threads) is the value; the reference's own
    shipped CPU renderer (tiled_renderer.rs restated, forward only, one
    thread, different semantics) is reported beside it.

    The same oracle run anchors the precision report: with gpu_view(sh_dtype,
    sh, v_rgba) -> (image RGBA, gradients) rendering and differentiating the
    view on the GPU, the FP32 and BF16-storage results are compared with the
    FP64 instantiation of the oracle (image PSNR and max |diff|, norm-wise
    gradient relative error; for BF16 against the stored, rounded SH and
    against the unrounded scene) and with the training target (PSNR)."""
    import torch

    from oracle import oracle as O

    cam = cams[0]
    t0 = time.perf_counter()
    f = O.Forward(scene.transforms, scene.sh, scene.raw_opacity, scene.sh_degree, cam)
    _, vp = O.loss(f.image, targets_np[0])
    f.backward(vp, mode=0)
    dt = time.perf_counter() - t0
    t1 = time.perf_counter()
    O.ref_cpu_forward(scene, cam)
    dt_ref = time.perf_counter() - t1
    out = {"value": dt * 1000.0, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
           "sample": "1 of the 8 views (1M Gaussians, 1280x720): oracle forward + loss + exact backward, "
                     "OpenMP over all host threads",
           "reference_cpu_forward": {"value": dt_ref * 1000.0, "unit": UNIT, "cores": 1,
                                     "sample": "the same view through the reference's shipped CPU renderer "
                                               "(TiledRenderer, forward only, single-threaded as shipped)"}}
    if gpu_view is None:
        return out
    tgt = targets_np[0]
    sh_bf = torch.as_tensor(scene.sh).to(torch.bfloat16).float().numpy()
    prec = {"view": "view 0 of the workload; upstream gradient = the oracle's loss gradient of that view"}
    for name, sh_gpu, sh_ref in (("f32", scene.sh, scene.sh), ("bf16_sh", scene.sh, sh_bf)):
        img, g = gpu_view("bf16" if name == "bf16_sh" else "f32", sh_gpu, vp)
        r64 = O.Forward(scene.transforms, sh_ref, scene.raw_opacity, scene.sh_degree, cam, f64=True)
        g64 = r64.backward(vp.astype(np.float64), mode=0)
        e = {"image_psnr_vs_fp64_db": _psnr(img[..., :3], r64.image[..., :3]),
             "image_max_abs_vs_fp64": float(np.abs(img - r64.image).max()),
             "grad_rel_err_vs_fp64": _grad_rel(g, g64),
             "psnr_vs_target_db": _psnr(img[..., :3], tgt)}
        if name == "bf16_sh":
            u64 = O.Forward(scene.transforms, scene.sh, scene.raw_opacity, scene.sh_degree, cam, f64=True)
            e["grad_rel_err_vs_fp64_unrounded_scene"] = _grad_rel(g, u64.backward(vp.astype(np.float64), mode=0))
        prec[name] = e
    prec["bf16_psnr_loss_vs_target_db"] = prec["f32"]["psnr_vs_target_db"] - prec["bf16_sh"]["psnr_vs_target_db"]
    out["precision"] = prec
    return out


def run_reference(args):
    """CPU reference arm: the oracle restatement of the reference's path on the host cores."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    from rustscan_b200 import scenes as S

    sc = S.config3(n=args.n, views=args.views)
    gt = S.config3_targets(n=args.n)
    gts = S.Scene(gt[0], gt[1], gt[2], 3, sc.cameras)
    cams = sc.cameras
    targets = {}

    def step(i):
        v = i % len(cams)
        if v not in targets:
            targets[v] = O.Forward(gts.transforms, gts.sh, gts.raw_opacity, 3, cams[v]).image[..., :3].copy()
        f = O.Forward(sc.transforms, sc.sh, sc.raw_opacity, sc.sh_degree, cams[v])
        _, vp = O.loss(f.image, targets[v])
        f.backward(vp, mode=0)

    for i in range(args.warmup):
        step(i)
    for i in range(args.warmup, args.warmup + args.steps):  # targets outside the timed region
        v = i % len(cams)
        if v not in targets:
            targets[v] = O.Forward(gts.transforms, gts.sh, gts.raw_opacity, 3, cams[v]).image[..., :3].copy()
    t0 = time.perf_counter()
    for i in range(args.warmup, args.warmup + args.steps):
        step(i)
    ms = (time.perf_counter() - t0) * 1000.0 / args.steps
    line = {"impl": "reference", "metric": METRIC, "value": ms, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded; see rustscan_b200/scenes.py)",
            "config": {"workload": "one view per step of " + WORKLOAD, "n_gaussians": args.n,
                       "resolution": "1280x720", "sh_degree": 3},
            "cpu_baseline": {"value": ms, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                             "sample": "one 1280x720 view per step: oracle forward + loss + exact backward"},
            "e2e": {"value": ms, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def profile_step(args):
    """Warm-up steps, then one batched step without a graph: every kernel of
    the step appears once in a profiler's launch list after the warm-up."""
    import torch

    from rustscan_b200 import LearningRates, Trainer, host_splats_to_device
    from rustscan_b200 import scenes as S

    sc = S.config3(n=args.n, views=args.views)
    cams = sc.cameras
    H, W = cams[0].height, cams[0].width
    # The tile shape and raster batch the autotuner picks on this workload.
    ctx = make_context(args.n, len(cams), tile=(16, 16), batch=128)
    splats = host_splats_to_device(sc)
    fit_capacity(ctx, splats, cams)
    rng = np.random.default_rng(0)
    targets = torch.as_tensor(rng.uniform(0, 1, (len(cams), H, W, 3)).astype(np.float32), device="cuda")
    tr = Trainer(ctx, splats, LearningRates(), use_graph=False)
    for i in range(args.warmup + 1):
        tr.train_step(cams, targets, i + 1)
    torch.cuda.synchronize()
    ctx.sync_status()
    print(json.dumps({"profile_step": "done", "views": len(cams), "n": args.n}), flush=True)


def _time_device(fn, steps, warmup):
    """Mean device ms of fn() over `steps` calls after `warmup`, CUDA events on the current stream."""
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        fn()
    e1.record(st)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def _render_op_line(args, name, sc, contexts, workload, dtype, extra=None):
    """fwd+bwd ms/view of the render op (gsr_render_forward + gsr_render_backward,
    one view per call, an N(0,1) upstream image gradient) for each named context
    configuration; the first is the headline of the line. End to end: the
    upstream gradient crosses from pinned host memory and the image comes back
    each step."""
    import torch

    from rustscan_b200 import Context, host_splats_to_device
    from rustscan_b200 import scenes as S

    cam = sc.cameras[0]
    H, W = cam.height, cam.width
    up = torch.as_tensor(S.upstream_grad(H, W), device="cuda")
    res = {}
    first = None
    for label, kw in contexts:
        ctx = Context(max_splats=sc.n, max_pixels=W * H, max_isects=kw.pop("max_isects", 16 << 20), **kw)
        splats = host_splats_to_device(sc, sh_dtype=torch.bfloat16 if kw.get("sh_dtype") == "bf16" else torch.float32)
        fit_capacity(ctx, splats, [cam])

        def step():
            ctx.render_forward(splats, [cam], check=False)
            ctx.render_backward(splats, up, stats=True)

        ms = _time_device(step, args.steps, args.warmup)
        res[label] = {"ms_per_view": ms, "stages_ms": stage_profile(ctx, step)}
        if first is None:
            first = (label, ctx, splats, ms)
        else:
            ctx.close()
    label, ctx, splats, ms = first
    up_h = torch.empty_like(up, device="cpu").pin_memory()
    up_h.copy_(up.cpu())
    img_h = torch.empty((H, W, 4), dtype=torch.float32).pin_memory()
    up_d = torch.empty_like(up)

    def e2e_step():
        up_d.copy_(up_h, non_blocking=True)
        _, imgs, _ = ctx.render_forward(splats, [cam], check=False)
        ctx.render_backward(splats, up_d, stats=True)
        img_h.copy_(imgs[0], non_blocking=True)

    ms_e2e = _time_device(e2e_step, args.steps, args.warmup)
    counts = ctx.export(0, "counts")
    evals = int(ctx.export(0, "nvisit").astype(np.int64).sum())
    ctx.close()
    line = {"metric": METRIC, "value": ms, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
            "data": "synthetic (seeded; see rustscan_b200/scenes.py)",
            "config": {"workload": workload, "n_gaussians": sc.n, "resolution": f"{W}x{H}", "sh_degree": sc.sh_degree,
                       "visible": int(counts[0]), "intersections": int(counts[1]), "headline": label},
            "paths_ms_per_view": res, "gaussian_pixel_evals_per_view": evals,
            "gaussian_pixel_evals_per_s": evals / (ms * 1e-3),
            "e2e": {"value": ms_e2e, "unit": UNIT, "h2d_bytes_per_step": int(up.numel() * 4),
                    "d2h_bytes_per_step": int(H * W * 16),
                    "inputs": "upstream image gradient from pinned host memory; rendered image read back"},
            "gpu_launches": None}
    if extra:
        line.update(extra)
    return line


def bench_config1(args):
    """Config 1: plain FP32 forward + backward of one 256x256 view (16,384
    Gaussians, SH degree 0), beside the CPU path on the same view."""
    from oracle import oracle as O
    from rustscan_b200 import scenes as S

    sc = S.config1()
    line = _render_op_line(args, "c1", sc, [("f32", {})],
                           "plain FP32 forward+backward, single view: 16,384 Gaussians, SH degree 0, 256x256", "f32")
    cam = sc.cameras[0]
    up = S.upstream_grad(cam.height, cam.width)
    reps = 20
    t0 = time.perf_counter()
    for _ in range(reps):
        O.Forward(sc.transforms, sc.sh, sc.raw_opacity, 0, cam).backward(up, mode=0)
    cpu_ms = (time.perf_counter() - t0) * 1000.0 / reps
    t1 = time.perf_counter()
    for _ in range(reps):
        O.ref_cpu_forward(sc, cam)
    ref_ms = (time.perf_counter() - t1) * 1000.0 / reps
    line["cpu_baseline"] = {"value": cpu_ms, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                            "sample": f"the same view, {reps} repetitions: oracle forward + exact backward, OpenMP over "
                                      "all host threads",
                            "reference_cpu_forward": {"value": ref_ms, "unit": UNIT, "cores": 1,
                                                      "sample": "the reference's shipped CPU renderer (forward only)"}}
    return line


def bench_config4(args):
    """Config 4: 3M Gaussians (5% flattened), one 1920x1080 view, fx = 1400:
    forward + backward with BF16 SH storage and the FP64 conic (the headline)
    beside plain FP32; precision of both against the FP64 oracle."""
    import torch

    from oracle import oracle as O
    from rustscan_b200 import Context, host_splats_to_device
    from rustscan_b200 import scenes as S

    sc = S.config4()
    line = _render_op_line(args, "c4", sc, [("bf16_sh_fp64_conic", {"sh_dtype": "bf16", "fp64_conic": True,
                                                                     "max_isects": 48 << 20}),
                                            ("f32", {"max_isects": 48 << 20})],
                           "mixed-precision render+backward: 3,000,000 Gaussians (5% flattened), SH degree 3, "
                           "1920x1080", "bf16 storage, f32 blend")
    if args.no_precision:
        return line
    cam = sc.cameras[0]
    up = S.upstream_grad(cam.height, cam.width)
    sh_bf = torch.as_tensor(sc.sh).to(torch.bfloat16).float().numpy()
    prec = {}
    t0 = time.perf_counter()
    u64 = O.Forward(sc.transforms, sc.sh, sc.raw_opacity, 3, cam, f64=True)
    g_u64 = u64.backward(up.astype(np.float64), mode=0)
    oracle_s = time.perf_counter() - t0
    for name, kw, sh_ref in (("f32", {}, None), ("bf16_sh_fp64_conic", {"sh_dtype": "bf16", "fp64_conic": True}, sh_bf)):
        ctx = Context(max_splats=sc.n, max_pixels=cam.width * cam.height, max_isects=48 << 20, **kw)
        sp = host_splats_to_device(sc, sh_dtype=torch.bfloat16 if kw.get("sh_dtype") == "bf16" else torch.float32)
        fit_capacity(ctx, sp, [cam])
        _, imgs, _ = ctx.render_forward(sp, [cam])
        g = ctx.render_backward(sp, torch.as_tensor(up, device="cuda"), stats=False)
        torch.cuda.synchronize()
        img = imgs[0].cpu().numpy()
        gg = {k: g[k].cpu().numpy() for k in ("v_transforms", "v_sh", "v_raw_opacity")}
        ctx.close()
        e = {"image_psnr_vs_fp64_db": _psnr(img[..., :3], u64.image[..., :3]),
             "image_max_abs_vs_fp64": float(np.abs(img - u64.image).max()),
             "grad_rel_err_vs_fp64": _grad_rel(gg, g_u64)}
        if sh_ref is not None:
            r64 = O.Forward(sc.transforms, sh_ref, sc.raw_opacity, 3, cam, f64=True)
            e["image_psnr_vs_fp64_of_stored_params_db"] = _psnr(img[..., :3], r64.image[..., :3])
            e["grad_rel_err_vs_fp64_of_stored_params"] = _grad_rel(gg, r64.backward(up.astype(np.float64), mode=0))
            del r64
        prec[name] = e
    prec["against"] = ("the FP64 oracle of the scene as given (unrounded parameters); for BF16 also the FP64 oracle "
                       "of the stored, BF16-rounded SH")
    prec["oracle_fp64_seconds"] = oracle_s
    line["precision"] = prec
    return line


def bench_config5(args):
    """Config 5: 32 views of mixed resolution over 2M Gaussians (BF16 SH
    storage), tile shape and raster batch from the autotuner: the batched
    training step (one launch per stage over all views, graph-replayed)
    against the plain single-view path (one view per call, no graph), per
    view; plus the batched step in FP32."""
    import torch

    from rustscan_b200 import Context, LearningRates, Trainer, autotune, host_splats_to_device
    from rustscan_b200 import scenes as S

    sc = S.config5()
    cams = sc.cameras
    nv = len(cams)
    pmax = max(c.width * c.height for c in cams)
    splats = host_splats_to_device(sc, sh_dtype=torch.bfloat16)
    tuned = autotune(splats, cams, reps=1, max_pixels=pmax, max_isects=24 << 20, sh_dtype="bf16")
    tile, batch = tuned["tile"], tuned["batch"]
    rng = np.random.default_rng(5)
    targets = torch.as_tensor(np.concatenate([rng.uniform(0, 1, c.width * c.height * 3) for c in cams])
                              .astype(np.float32), device="cuda")
    offs = np.concatenate([[0], np.cumsum([c.width * c.height * 3 for c in cams])])

    def batched_ms(sh_dtype, sp):
        ctx = Context(max_splats=sc.n, max_views=nv, max_pixels=pmax, max_isects=24 << 20, sh_dtype=sh_dtype,
                      tile=tile, batch=batch)
        fit_capacity(ctx, sp, cams)
        counts = [ctx.export(v, "counts") for v in range(nv)]
        tr = Trainer(ctx, sp, LearningRates(), total_iterations=30000, use_graph=True)
        ms = time_steps(lambda it: tr.train_step(cams, targets, it), args.steps, args.warmup, 1)
        stages = stage_profile(ctx, lambda: Trainer(ctx, sp, LearningRates(), use_graph=False).train_step(
            cams, targets, args.warmup + args.steps + 1))
        ctx.close()
        return ms / args.steps / nv, counts, stages

    ms_b, counts, stages = batched_ms("bf16", splats)
    # Plain path: one view per call, in a context sized for one view.
    ctx1 = Context(max_splats=sc.n, max_views=1, max_pixels=pmax, max_isects=24 << 20, sh_dtype="bf16", tile=tile,
                   batch=batch)
    fit_capacity(ctx1, splats, [max(cams, key=lambda c: c.width * c.height)])
    tr1 = Trainer(ctx1, splats, LearningRates(), use_graph=False)
    per_view = []
    for v, cam in enumerate(cams):
        fit_capacity(ctx1, splats, [cam])
        tv = targets[offs[v]:offs[v + 1]]
        per_view.append(time_steps(lambda it: tr1.train_step([cam], tv, it), max(2, args.steps // 2), 1, 1)
                        / max(2, args.steps // 2))
    ctx1.close()
    splats32 = host_splats_to_device(sc)
    ms_f32, _, _ = batched_ms("f32", splats32)
    V = [int(c[0]) for c in counts]
    I = [int(c[1]) for c in counts]
    plain = float(np.mean(per_view))
    return {"metric": METRIC, "value": ms_b, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_b * nv, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16 storage, f32 blend", "data": "synthetic (seeded; see rustscan_b200/scenes.py)",
            "config": {"workload": "uneven batch: 32 views of mixed resolution (320x240 to 1920x1080), 2,000,000 "
                                   "Gaussians, SH degree 3, BF16 SH storage, one training step over all views",
                       "resolutions": [f"{c.width}x{c.height}" for c in cams], "visible_per_view": V,
                       "intersections_per_view": I, "tile": f"{tile[0]}x{tile[1]}", "raster_batch": batch,
                       "tile_and_batch": "autotuner (gsr_autotune)", "graph": True},
            "plain_single_view_ms_per_view": plain, "plain_per_view_ms": per_view,
            "batched_over_plain": ms_b / plain, "f32_batched_ms_per_view": ms_f32,
            "stages_ms_per_step": stages, "gpu_launches": None}


def main():
    args = parse()
    if args.config != "c3":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference arm is timed on the c3 workload"}))
            return
        import torch

        torch.cuda.set_device(0)
        fn = {"c1": bench_config1, "c4": bench_config4, "c5": bench_config5}[args.config]
        print(json.dumps(fn(args)), flush=True)
        return
    if args.impl == "reference":
        run_reference(args)
        return
    import torch

    from rustscan_b200 import LearningRates, Trainer, host_splats_to_device
    from rustscan_b200 import scenes as S

    world, rank, local = dist_setup(args)
    if args.mode == "profile":
        profile_step(args)
        return
    sc = S.config3(seed_offset=rank, n=args.n, views=args.views)
    gt_tr, gt_sh, gt_op = S.config3_targets(seed_offset=rank, n=args.n)
    cams = sc.cameras
    nv = len(cams)
    H, W = cams[0].height, cams[0].width

    # Tile shape and raster batch from the autotuner (untimed), as a user
    # would pick them for this scene and view mix.
    from rustscan_b200 import autotune

    splats = host_splats_to_device(sc)
    tuned = autotune(splats, cams, reps=2, max_pixels=W * H, max_isects=24 << 20)
    tile, batch = tuned["tile"], tuned["batch"]

    # Targets: renders of the hidden ground-truth set.
    ctx = make_context(args.n, nv, tile=tile, batch=batch)
    gts = host_splats_to_device(S.Scene(gt_tr, gt_sh, gt_op, 3, cams))
    fit_capacity(ctx, gts, cams)
    flat, _, _ = ctx.render_forward(gts, cams)
    # The training frames are 8-bit RGB images (what a camera or the dataset
    # decoder gives); the device targets are their conversion on the GPU.
    frames_u8 = (flat.view(nv, H, W, 4)[..., :3].clamp(0, 1) * 255.0).round().to(torch.uint8).contiguous()
    targets = ctx.frames_to_targets(frames_u8.view(-1), [(v * H * W * 3, W, H) for v in range(nv)],
                                    cams).view(nv, H, W, 3)
    del gts
    fit_capacity(ctx, splats, cams)
    counts = [ctx.export(v, "counts") for v in range(nv)]
    V = [int(c[0]) for c in counts]
    I = [int(c[1]) for c in counts]
    P = H * W

    # ---- batched, graph-replayed training step -----------------------------
    trainer = Trainer(ctx, splats, LearningRates(), total_iterations=30000, use_graph=True)

    def batched(it):
        trainer.train_step(cams, targets, it)

    for i in range(args.warmup):
        batched(i + 1)
    torch.cuda.synchronize()
    ctx.sync_status()
    with Clocks(local) as clk:
        ms_total = time_steps(batched, args.steps, 0, world)
    ms_step = ms_total / args.steps
    value = ms_step / nv
    kernels_per_step = int(ctx._lib.gsr_graph_kernel_count(ctx._h))

    # ---- stage profile of one (non-graph) batched step: roofline ---------------
    tr_prof = Trainer(ctx, splats, LearningRates(), use_graph=False)
    tr_prof.opt = trainer.opt
    stages = stage_profile(ctx, lambda: tr_prof.train_step(cams, targets, args.warmup + args.steps + 1))
    hbm, peak_kind = peaks()
    # Gaussian-pixel evaluations of the step's forward: per pixel, the list
    # entries up to its termination (the reference's blend loop count).
    evals_per_step = sum(int(ctx.export(v, "nvisit").astype(np.int64).sum()) for v in range(nv))
    # Algorithmic bytes per launch (all views of the step).
    algo = {
        "raster_fwd": sum(40 * I[v] + 16 * P for v in range(nv)),
        "raster_bwd": sum(40 * I[v] + 32 * P + 56 * V[v] for v in range(nv)),
        "tile_sort": sum(16 * I[v] for v in range(nv)),  # two passes over packed 4-byte keys, read + write
        "project": 44 * args.n + sum((12 + 48 + 192) * V[v] for v in range(nv)),
        "adam": 28 * (10 + 48 + 1) * args.n + 8 * 10 * args.n,
    }
    dom = max((k for k in algo), key=lambda k: stages.get(k, 0.0))
    achieved = algo[dom] / (stages[dom] * 1e-3) / 1e9
    # DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) from one ncu
    # capture of a single 1280x720 view of this workload (6,273,269
    # intersections), scaled to the launch by its intersections (the raster
    # and tile-sort traffic grows with them) or, for Adam, taken as is (it
    # sweeps the N parameters once per step).
    traffic_coeff = {"raster_bwd": (37.736e6 + 0.016e6) / 6273269, "raster_fwd": (14.121e6 + 0.219e6) / 6273269,
                     "tile_sort": (30.3e6 + 0.4e6 + 30.4e6 + 0.6e6) / 6273269}
    if dom in traffic_coeff:
        traffic = traffic_coeff[dom] * sum(I)
    elif dom == "adam":
        traffic = (160.0e6 + 63.1e6 + 768.0e6 + 520.4e6 + 16.0e6) * args.n / 1_000_000
    else:
        traffic = None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "traffic": traffic, "peak_kind": peak_kind,
                "algorithmic_bytes": algo[dom], "launch_ms": stages[dom],
                "traffic_over_algorithmic": (traffic / algo[dom]) if traffic else None}
    # The raster kernels are bound by instruction issue, not by HBM: their
    # issue roofline is the SMs' warp-instruction issue rate (4 schedulers
    # per SM, one warp instruction each per clock) at the SM clock measured
    # during the timed region. The warp instructions per launch come from
    # one ncu capture of a single 1280x720 view (smsp__inst_executed.sum),
    # scaled to the launch by its intersections.
    inst_per_isect = {"raster_bwd": WARP_INST_PER_ISECT["raster_bwd"], "raster_fwd": WARP_INST_PER_ISECT["raster_fwd"]}
    sm_mhz = clk.summary().get("sm_mhz") or 1965.0
    n_sm = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    if dom in inst_per_isect:
        winst = inst_per_isect[dom] * sum(I)
        peak_issue = n_sm * 4 * sm_mhz * 1e6
        roofline["issue"] = {"bound": "issue", "achieved": winst / (stages[dom] * 1e-3) / 1e9,
                             "peak": peak_issue / 1e9, "unit": "G warp-instructions/s",
                             "frac": winst / (stages[dom] * 1e-3) / peak_issue, "warp_instructions": winst,
                             "sm_mhz": sm_mhz, "sms": n_sm,
                             "source": "warp instructions per intersection from ncu smsp__inst_executed.sum on one "
                                       "view, times this launch's intersections"}

    # ---- the same batched step with BF16 SH storage ---------------------------
    bf16_ms = None
    if not args.no_bf16:
        ctx_b = make_context(args.n, nv, sh_dtype="bf16", tile=tile, batch=batch)
        splats_b = host_splats_to_device(sc, sh_dtype=torch.bfloat16)
        fit_capacity(ctx_b, splats_b, cams)
        trainer_b = Trainer(ctx_b, splats_b, LearningRates(), total_iterations=30000, use_graph=True)
        bf16_ms = time_steps(lambda it: trainer_b.train_step(cams, targets, it), args.steps, args.warmup,
                             world) / args.steps / nv
        del trainer_b, splats_b
        ctx_b.close()

    # ---- plain single-view path (one view per call, FP32, no graph) ------------
    plain = None
    if not args.no_plain:
        ctx1 = make_context(args.n, 1, tile=tile, batch=batch)
        fit_capacity(ctx1, splats, [cams[0]])
        tr1 = Trainer(ctx1, splats, LearningRates(), use_graph=False)

        def plain_step(it):
            v = (it - 1) % nv
            tr1.train_step([cams[v]], targets[v], it)

        ms1 = time_steps(plain_step, args.steps, args.warmup, world)
        plain = ms1 / args.steps
        ctx1.close()

    # ---- end to end through the public API with host buffers -------------------
    # The step's inputs are the views' 8-bit frames in pinned host memory;
    # Trainer.train_step_frames uploads them and converts them on the device.
    host_frames = [torch.empty((H, W, 3), dtype=torch.uint8, pin_memory=True) for _ in range(nv)]
    for v in range(nv):
        host_frames[v].copy_(frames_u8[v].cpu())
    host_loss = torch.empty(nv, dtype=torch.float32, pin_memory=True)
    e2e_warm = 1

    def e2e_step(it):
        # Each timed step's frames cross PCIe once: the first timed step
        # copies its own, every other one was prefetched by the step before
        # it (inside the timed region); the warm-up and the last timed step
        # prefetch nothing.
        nxt = host_frames if e2e_warm < it < e2e_warm + args.steps else None
        loss = trainer.train_step_frames(cams, host_frames, it, next_frames=nxt)
        host_loss.copy_(loss, non_blocking=True)

    ms_e2e = time_steps(e2e_step, args.steps, e2e_warm, world) / args.steps
    e2e = {"value": ms_e2e / nv, "unit": UNIT, "h2d_bytes_per_step": int(sum(f.numel() for f in host_frames)),
           "d2h_bytes_per_step": int(nv * 4), "inputs": "8-bit RGB frames, converted to f32 targets on the device"}

    def gpu_view(sh_dtype, sh, v_rgba):
        # View 0 rendered and differentiated on the GPU from the scene's own
        # (unstepped) parameters, for the precision report.
        cp = make_context(args.n, 1, sh_dtype=sh_dtype, tile=tile, batch=batch)
        sp = host_splats_to_device(S.Scene(sc.transforms, sh, sc.raw_opacity, sc.sh_degree, [cams[0]]),
                                   sh_dtype=torch.bfloat16 if sh_dtype == "bf16" else torch.float32)
        fit_capacity(cp, sp, [cams[0]])
        _, imgs, _ = cp.render_forward(sp, [cams[0]])
        g = cp.render_backward(sp, torch.as_tensor(np.ascontiguousarray(v_rgba), device="cuda"))
        torch.cuda.synchronize()
        res = imgs[0].cpu().numpy(), {k: g[k].cpu().numpy() for k in ("v_transforms", "v_sh", "v_raw_opacity")}
        cp.close()
        return res

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(sc, cams, targets.cpu().numpy(), None if args.no_precision else gpu_view)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded; see rustscan_b200/scenes.py)",
            "config": {"workload": WORKLOAD, "n_gaussians": args.n, "views_per_step": nv, "resolution": f"{W}x{H}",
                       "sh_degree": 3, "sh_storage": "f32", "tile": f"{tile[0]}x{tile[1]}",
                       "raster_batch": batch, "tile_and_batch": "autotuner (gsr_autotune)",
                       "loss": "0.8 L1 + 0.2 D-SSIM", "optimizer": "Adam (lr_pos 1.6e-4)", "graph": True,
                       "l2": "inputs larger than L2 (params 236 MB + 8 views of state per step)",
                       "visible_per_view": V, "intersections_per_view": I, "parallelism": "replicas" if world > 1 else "1 GPU"},
            "plain_single_view_ms_per_view": plain,
            "bf16_sh_batched_ms_per_view": bf16_ms,
            "gaussian_pixel_evals_per_step": evals_per_step,
            "gaussian_pixel_evals_per_s": evals_per_step / (ms_step * 1e-3),
            "precision": (cpu or {}).pop("precision", None),
            "stages_ms_per_step": stages,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": kernels_per_step * args.steps,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
