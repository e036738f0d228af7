"""Seeded synthetic scenes for the rasterizer workloads.

Every workload is a seeded restatement of a benchmark configuration (there is
no dataset on this path): Gaussians in the RustGS packed layout
(``transforms [N,10]`` = position xyz + quaternion wxyz + log-scale xyz,
``sh [N,K,3]`` coefficient-major, ``raw_opacity [N]`` logits;
RustGS/src/training/engine/splats.rs:7-18) and pinhole cameras with a
column-major world->camera matrix (RustGS/src/core/camera.rs:30-37, +Z
forward, +Y down, principal point in pixels).

The generator is numpy's PCG64 seeded with ``0x6A5C0DE + index``; normals come
from numpy's standard-normal sampler. Nothing here touches a GPU.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

SH_C0 = 0.28209479177387814  # helpers.wgsl:5
SEED_BASE = 0x6A5C0DE


@dataclasses.dataclass
class Camera:
    """Pinhole camera; field layout matches ``gsr_camera`` in include/gsr.h."""

    viewmat: np.ndarray  # (16,) float32, column-major world->camera
    fx: float
    fy: float
    cx: float
    cy: float
    width: int
    height: int
    campos: np.ndarray  # (3,) float32 camera centre in world space

    def as_record(self) -> np.ndarray:
        """Pack into the 28-word ``gsr_camera`` record (float32 view)."""
        rec = np.zeros(28, dtype=np.float32)
        rec[0:16] = self.viewmat
        rec[16:20] = (self.fx, self.fy, self.cx, self.cy)
        rec.view(np.uint32)[20] = self.width
        rec.view(np.uint32)[21] = self.height
        rec[22:25] = self.campos
        return rec


def camera_from_rt(R: np.ndarray, t: np.ndarray, fx, fy, cx, cy, width, height) -> Camera:
    """World->camera rotation ``R`` (rows are camera axes) and translation ``t``."""
    M = np.eye(4, dtype=np.float64)
    M[:3, :3] = R
    M[:3, 3] = t
    viewmat = M.T.reshape(-1).astype(np.float32)  # column-major
    campos = (-R.T @ t).astype(np.float32)
    return Camera(viewmat, float(fx), float(fy), float(cx), float(cy), int(width), int(height), campos)


def look_at(eye, target, fx, fy, cx, cy, width, height, up=(0.0, 1.0, 0.0)) -> Camera:
    """Camera at ``eye`` looking at ``target`` (x right, y down, z forward)."""
    eye = np.asarray(eye, dtype=np.float64)
    z = np.asarray(target, dtype=np.float64) - eye
    z /= np.linalg.norm(z)
    u = np.asarray(up, dtype=np.float64)
    if abs(float(np.dot(u, z))) > 0.999:
        u = np.array([1.0, 0.0, 0.0])
    x = np.cross(z, u)
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    R = np.stack([x, y, z], axis=0)
    return camera_from_rt(R, -R @ eye, fx, fy, cx, cy, width, height)


@dataclasses.dataclass
class Scene:
    transforms: np.ndarray  # [N,10] float32
    sh: np.ndarray  # [N,K,3] float32
    raw_opacity: np.ndarray  # [N] float32
    sh_degree: int
    cameras: list
    name: str = ""

    @property
    def n(self) -> int:
        return int(self.raw_opacity.shape[0])


def _quats(rng, n):
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return q


def _gaussians(rng, n, degree, means, logscale_mu=-4.0, logscale_sigma=0.5, hi_sigma=0.05):
    K = (degree + 1) ** 2
    tr = np.empty((n, 10), dtype=np.float32)
    tr[:, 0:3] = means
    tr[:, 3:7] = _quats(rng, n)
    tr[:, 7:10] = rng.normal(logscale_mu, logscale_sigma, (n, 3))
    sh = np.zeros((n, K, 3), dtype=np.float32)
    rgb = rng.uniform(0.0, 1.0, (n, 3))
    sh[:, 0, :] = (rgb - 0.5) / SH_C0
    if K > 1:
        sh[:, 1:, :] = rng.normal(0.0, hi_sigma, (n, K - 1, 3))
    opac = rng.standard_normal(n).astype(np.float32)
    return tr, sh, opac


def _blob_means(rng, n, blobs=8, sigma=0.3, cube=4.0):
    centres = rng.uniform(-cube / 2, cube / 2, (blobs, 3))
    which = rng.integers(0, blobs, n)
    return centres[which] + rng.normal(0.0, sigma, (n, 3))


def _sphere_dirs(rng, k):
    d = rng.standard_normal((k, 3))
    return d / np.linalg.norm(d, axis=1, keepdims=True)


def config1(seed_offset=0, n=16384):
    """Plain FP32 single view: 16,384 Gaussians, SH degree 0, 256x256."""
    rng = np.random.Generator(np.random.PCG64(SEED_BASE + 0 + seed_offset))
    means = rng.uniform(-1.0, 1.0, (n, 3))
    tr, sh, op = _gaussians(rng, n, 0, means)
    cam = camera_from_rt(np.eye(3), np.array([0.0, 0.0, 3.0]), 256, 256, 128, 128, 256, 256)
    return Scene(tr, sh, op, 0, [cam], "c1")


def config2(seed_offset=0, n=200_000):
    """Adjoint check: 200k Gaussians in 8 blobs, SH degree 3, 640x480."""
    rng = np.random.Generator(np.random.PCG64(SEED_BASE + 1 + seed_offset))
    tr, sh, op = _gaussians(rng, n, 3, _blob_means(rng, n))
    cam = camera_from_rt(np.eye(3), np.array([0.0, 0.0, 5.0]), 525, 525, 319.5, 239.5, 640, 480)
    return Scene(tr, sh, op, 3, [cam], "c2")


def config3(seed_offset=0, n=1_000_000, views=8, width=1280, height=720, focal=1050.0):
    """Batched step: 1M Gaussians, SH degree 3, 8 views of 1280x720 on a radius-4 sphere."""
    rng = np.random.Generator(np.random.PCG64(SEED_BASE + 2 + seed_offset))
    tr, sh, op = _gaussians(rng, n, 3, _blob_means(rng, n))
    cams = [
        look_at(4.0 * d, (0, 0, 0), focal, focal, (width - 1) / 2, (height - 1) / 2, width, height)
        for d in _sphere_dirs(rng, views)
    ]
    return Scene(tr, sh, op, 3, cams, "c3")


def config3_targets(seed_offset=0, n=1_000_000):
    """The hidden ground-truth Gaussian set whose renders are config 3's targets."""
    rng = np.random.Generator(np.random.PCG64(SEED_BASE + 102 + seed_offset))
    tr, sh, op = _gaussians(rng, n, 3, _blob_means(np.random.Generator(np.random.PCG64(SEED_BASE + 2 + seed_offset)), n))
    return tr, sh, op


def config4(seed_offset=0, n=3_000_000, width=1920, height=1080):
    """Mixed precision: 3M Gaussians, 5% flattened (one log-scale -9), 1920x1080
    (fx = fy = 1400 at full width; scaled with the width for smaller cases)."""
    rng = np.random.Generator(np.random.PCG64(SEED_BASE + 3 + seed_offset))
    tr, sh, op = _gaussians(rng, n, 3, _blob_means(rng, n))
    flat = rng.random(n) < 0.05
    axis = rng.integers(0, 3, n)
    tr[np.nonzero(flat)[0], 7 + axis[flat]] = -9.0
    f = 1400.0 * width / 1920.0
    cam = look_at(np.array([0.0, 0.0, -5.0]), (0, 0, 0), f, f, (width - 1) / 2, (height - 1) / 2, width, height)
    return Scene(tr, sh, op, 3, [cam], "c4")


C5_RESOLUTIONS = ((320, 240), (640, 480), (1280, 720), (1920, 1080))


def config5(seed_offset=0, n=2_000_000, views=32, resolutions=C5_RESOLUTIONS):
    """Uneven batch: 32 views of mixed resolution at distances U[1.5, 8]."""
    rng = np.random.Generator(np.random.PCG64(SEED_BASE + 4 + seed_offset))
    tr, sh, op = _gaussians(rng, n, 3, _blob_means(rng, n))
    res = list(resolutions)
    cams = []
    for d in _sphere_dirs(rng, views):
        w, h = res[int(rng.integers(0, len(res)))]
        r = float(rng.uniform(1.5, 8.0))
        f = 0.8203125 * w
        cams.append(look_at(r * d, (0, 0, 0), f, f, (w - 1) / 2, (h - 1) / 2, w, h))
    return Scene(tr, sh, op, 3, cams, "c5")


def small_scene(n=2000, degree=3, width=96, height=80, seed=7, views=1, blobs=True, logscale_mu=-3.0):
    """Small seeded scene for parity tests the CPU oracle finishes in well under a second."""
    rng = np.random.Generator(np.random.PCG64(SEED_BASE + 1000 + seed))
    means = _blob_means(rng, n, blobs=4, sigma=0.4, cube=2.0) if blobs else rng.uniform(-1, 1, (n, 3))
    tr, sh, op = _gaussians(rng, n, degree, means, logscale_mu=logscale_mu)
    f = 0.9 * width
    cams = [
        look_at(3.5 * d, (0, 0, 0), f, f * 1.05, width / 2 - 0.25, height / 2 + 0.5, width, height)
        for d in _sphere_dirs(rng, views)
    ]
    return Scene(tr, sh, op, degree, cams, f"small{seed}")


def upstream_grad(height, width, seed=11):
    """N(0,1) upstream image gradient per RGB channel, zero for alpha."""
    rng = np.random.Generator(np.random.PCG64(SEED_BASE + 5000 + seed))
    g = np.zeros((height, width, 4), dtype=np.float32)
    g[..., :3] = rng.standard_normal((height, width, 3))
    return g


CONFIGS = {1: config1, 2: config2, 3: config3, 4: config4, 5: config5}


def tiles_for(width, height, tw=16, th=16):
    return math.ceil(width / tw), math.ceil(height / th)
