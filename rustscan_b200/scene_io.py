"""Scene files in the 3DGS property layout, mirroring RustGS/src/io/scene_io.rs.

* ``save_splats_ply`` / ``load_splats_ply`` (scene_io.rs:99-179, 485-557,
  639-797): vertex properties x y z nx ny nz f_dc_0..2 f_rest_0..44 opacity
  scale_0..2 rot_0..3. Written as ASCII with the reference's comments
  (iterations, final_loss, sh_degree, ``opacity_representation raw_logit``,
  ``sh_coeff_layout channel_major``), f_rest padded to 45 values. Read as
  ASCII or binary little endian, float or double properties; the opacity
  representation (default raw logit) and the f_rest layout (default channel
  major, i.e. all red coefficients, then green, then blue) come from the
  comments, the SH degree from ``comment sh_degree`` / ``comment SH degree:``
  or from the f_rest count.
* ``save_splats_splat`` / ``load_splats_splat`` (scene_io.rs:559-625,
  799-868): 32-byte rows of position (3 f32), scale (3 f32), RGBA (4 u8) and
  the normalised quaternion (4 u8, (q + 1) * 128); degree 0 only.
* ``save_splats`` / ``load_splats`` pick the format from the extension.

Scenes use this package's host layout: transforms [N,10] = position,
quaternion (w, x, y, z), log scale; SH [N,K,3] (coefficient-major, RGB
interleaved, as RustGS stores them); opacity logits [N].
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np

from .scenes import SH_C0, Scene


class SceneIoError(ValueError):
    pass


@dataclasses.dataclass
class SplatMetadata:
    iterations: int = 0
    final_loss: float = 0.0
    gaussian_count: int = 0
    sh_degree: int = 0


def _sh_count(degree: int) -> int:
    return (degree + 1) * (degree + 1)


def _logit(p):
    p = np.clip(np.asarray(p, np.float32), 1e-6, 1.0 - 1e-6)
    return np.log(p / (1.0 - p)).astype(np.float32)


def _fmt(x) -> str:
    # Shortest round-trip text of an f32 (the reference writes f32 Display).
    return np.format_float_positional(np.float32(x), unique=True, trim="-")


def save_splats_ply(path, scene: Scene, metadata: SplatMetadata | None = None) -> None:
    md = metadata or SplatMetadata(sh_degree=scene.sh_degree, gaussian_count=scene.n)
    tr = np.asarray(scene.transforms, np.float32)
    sh = np.asarray(scene.sh, np.float32).reshape(scene.n, -1, 3)
    op = np.asarray(scene.raw_opacity, np.float32)
    n = tr.shape[0]
    K = sh.shape[1]
    lines = ["ply", "format ascii 1.0", "comment Generated by RustGS", f"comment iterations {md.iterations}",
             f"comment final_loss {md.final_loss}", f"comment sh_degree {md.sh_degree}",
             "comment opacity_representation raw_logit", "comment sh_coeff_layout channel_major",
             f"element vertex {n}"]
    lines += [f"property float {p}" for p in ("x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2")]
    lines += [f"property float f_rest_{i}" for i in range(45)]
    lines += [f"property float {p}" for p in ("opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2",
                                              "rot_3")]
    lines.append("end_header")
    # f_rest channel major: rest[k][c] -> [c * (K-1) + k], padded to 45.
    rest = np.zeros((n, 45), np.float32)
    if K > 1:
        cm = sh[:, 1:, :].transpose(0, 2, 1).reshape(n, -1)
        rest[:, :cm.shape[1]] = cm[:, :45]
    body = []
    for i in range(n):
        vals = [tr[i, 0], tr[i, 1], tr[i, 2], 0, 0, 0, sh[i, 0, 0], sh[i, 0, 1], sh[i, 0, 2], *rest[i], op[i],
                tr[i, 7], tr[i, 8], tr[i, 9], tr[i, 3], tr[i, 4], tr[i, 5], tr[i, 6]]
        body.append(" ".join(_fmt(v) for v in vals))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
        f.write("\n".join(body) + ("\n" if body else ""))


def _parse_header(data: bytes):
    pos = 0
    hdr = dict(format="ascii", count=0, props=[], types=[], opacity=None, layout=None, md=SplatMetadata(),
               explicit_degree=False)
    first = True
    element = None
    while pos < len(data):
        end = data.find(b"\n", pos)
        end = len(data) if end < 0 else end + 1
        line = data[pos:end].decode("utf-8").strip()
        pos = end
        if first:
            if line != "ply":
                raise SceneIoError("missing PLY magic header")
            first = False
            continue
        if line.startswith("format "):
            f = line[len("format "):].strip()
            if f == "ascii 1.0":
                hdr["format"] = "ascii"
            elif f == "binary_little_endian 1.0":
                hdr["format"] = "binary"
            else:
                raise SceneIoError(f"unsupported PLY format {f}")
        elif line.startswith("comment iterations "):
            hdr["md"].iterations = int(line.split()[-1]) if line.split()[-1].isdigit() else 0
        elif line.startswith("comment final_loss "):
            try:
                hdr["md"].final_loss = float(line.split()[-1])
            except ValueError:
                hdr["md"].final_loss = 0.0
        elif line.startswith("comment sh_degree ") or line.startswith("comment SH degree: "):
            try:
                hdr["md"].sh_degree = int(line.split()[-1])
                hdr["explicit_degree"] = True
            except ValueError:
                pass
        elif line.startswith("comment opacity_representation "):
            hdr["opacity"] = {"probability": "probability", "raw_logit": "raw_logit"}.get(line.split()[-1])
        elif line.startswith("comment sh_coeff_layout "):
            hdr["layout"] = {"interleaved": "interleaved", "channel_major": "channel_major"}.get(line.split()[-1])
        elif line.startswith("element "):
            parts = line.split()
            element = parts[1] if len(parts) > 1 else ""
            if element == "vertex":
                hdr["count"] = int(parts[2]) if len(parts) > 2 else 0
        elif line.startswith("property ") and element == "vertex":
            parts = line.split()
            if len(parts) != 3:
                raise SceneIoError(f"invalid property declaration: {line}")
            if parts[1] not in ("float", "float32", "double", "float64"):
                raise SceneIoError(f"unsupported vertex property type {parts[1]}")
            hdr["types"].append("<f8" if parts[1] in ("double", "float64") else "<f4")
            hdr["props"].append(parts[2])
        elif line == "end_header":
            return hdr, pos
    raise SceneIoError("missing end_header")


def _infer_degree(explicit, degree, rest_count):
    if explicit:
        return degree
    if rest_count == 0:
        return 0
    if rest_count % 3:
        raise SceneIoError(f"invalid f_rest property count {rest_count}; expected a multiple of 3")
    per = rest_count // 3 + 1
    d = 0
    while _sh_count(d) < per:
        d += 1
    if _sh_count(d) != per:
        raise SceneIoError(f"could not infer SH degree from {rest_count} rest coefficients")
    return d


def load_splats_ply(path):
    data = open(path, "rb").read()
    hdr, off = _parse_header(data)
    props, n = hdr["props"], hdr["count"]

    def col(name):
        if name not in props:
            raise SceneIoError(f"missing required PLY property {name}")
        return props.index(name)

    if hdr["format"] == "binary":
        dt = np.dtype([(f"p{i}", t) for i, t in enumerate(hdr["types"])])
        need = dt.itemsize * n
        if len(data) - off < need:
            raise SceneIoError(f"binary PLY truncated: expected at least {need} bytes, got {len(data) - off}")
        rec = np.frombuffer(data, dtype=dt, count=n, offset=off)
        table = np.stack([rec[f"p{i}"].astype(np.float32) for i in range(len(props))], axis=1) if n else \
            np.zeros((0, len(props)), np.float32)
    else:
        text = data[off:].decode("utf-8").split()
        if len(text) < n * len(props):
            raise SceneIoError("ascii PLY truncated")
        table = np.asarray(text[:n * len(props)], dtype=np.float64).astype(np.float32).reshape(n, len(props))
    rest_idx = sorted(((int(p[len("f_rest_"):]), i) for i, p in enumerate(props) if p.startswith("f_rest_")))
    degree = _infer_degree(hdr["explicit_degree"], hdr["md"].sh_degree, len(rest_idx))
    K = _sh_count(degree)
    tr = np.zeros((n, 10), np.float32)
    tr[:, 0] = table[:, col("x")]
    tr[:, 1] = table[:, col("y")]
    tr[:, 2] = table[:, col("z")]
    for i in range(4):
        tr[:, 3 + i] = table[:, col(f"rot_{i}")]
    for i in range(3):
        tr[:, 7 + i] = table[:, col(f"scale_{i}")]
    opacity = table[:, col("opacity")]
    op = _logit(opacity) if hdr["opacity"] == "probability" else opacity.astype(np.float32)
    sh = np.zeros((n, K, 3), np.float32)
    for ch in range(3):
        sh[:, 0, ch] = table[:, col(f"f_dc_{ch}")]
    keep = (K - 1) * 3
    if keep > 0:
        rest = np.zeros((n, keep), np.float32)
        for dst, (_, src) in enumerate(rest_idx[:keep]):
            rest[:, dst] = table[:, src]
        if (hdr["layout"] or "channel_major") == "channel_major":
            sh[:, 1:, :] = rest.reshape(n, 3, K - 1).transpose(0, 2, 1)
        else:
            sh[:, 1:, :] = rest.reshape(n, K - 1, 3)
    md = hdr["md"]
    md.gaussian_count = n
    md.sh_degree = degree
    return Scene(tr, sh, op, degree, [], os.path.basename(str(path))), md


def _normalized_quat(q):
    q = np.asarray(q, np.float32)
    l2 = (q * q).sum(axis=1)
    ok = np.isfinite(l2) & (l2 > 1e-12)
    out = np.tile(np.array([1, 0, 0, 0], np.float32), (q.shape[0], 1))
    out[ok] = q[ok] * (np.float32(1) / np.sqrt(l2[ok]))[:, None]
    return out


def save_splats_splat(path, scene: Scene, metadata: SplatMetadata | None = None) -> None:
    tr = np.asarray(scene.transforms, np.float32)
    sh = np.asarray(scene.sh, np.float32).reshape(scene.n, -1, 3)
    n = tr.shape[0]
    rows = np.zeros(n, dtype=[("pos", "<f4", 3), ("scale", "<f4", 3), ("rgba", "u1", 4), ("rot", "u1", 4)])
    rows["pos"] = tr[:, 0:3]
    rows["scale"] = np.exp(tr[:, 7:10])
    rgb = sh[:, 0, :] * np.float32(SH_C0) + np.float32(0.5)
    opac = 1.0 / (1.0 + np.exp(-np.asarray(scene.raw_opacity, np.float32)))
    rgba = np.concatenate([rgb, opac[:, None]], axis=1)
    rows["rgba"] = np.round(np.clip(rgba, 0.0, 1.0) * 255.0).astype(np.uint8)
    q = _normalized_quat(tr[:, 3:7])
    rows["rot"] = np.clip(np.round(np.clip(q, -1.0, 1.0) * 128.0 + 128.0), 0, 255).astype(np.uint8)
    rows.tofile(path)


def load_splats_splat(path):
    data = open(path, "rb").read()
    if len(data) % 32:
        raise SceneIoError(f"invalid .splat byte length {len(data)}; expected a multiple of 32")
    rows = np.frombuffer(data, dtype=[("pos", "<f4", 3), ("scale", "<f4", 3), ("rgba", "u1", 4), ("rot", "u1", 4)])
    n = rows.shape[0]
    tr = np.zeros((n, 10), np.float32)
    tr[:, 0:3] = rows["pos"]
    tr[:, 7:10] = np.log(np.maximum(rows["scale"], np.float32(1e-8)))
    tr[:, 3:7] = _normalized_quat((rows["rot"].astype(np.float32) - 128.0) / 128.0)
    rgb = rows["rgba"][:, :3].astype(np.float32) / 255.0
    sh = ((rgb - 0.5) / np.float32(SH_C0)).astype(np.float32).reshape(n, 1, 3)
    op = _logit(rows["rgba"][:, 3].astype(np.float32) / 255.0)
    return Scene(tr, sh, op, 0, [], os.path.basename(str(path))), SplatMetadata(0, 0.0, n, 0)


def _format(path):
    ext = os.path.splitext(str(path))[1].lower()
    if ext == ".ply":
        return "ply"
    if ext == ".splat":
        return "splat"
    if ext:
        raise SceneIoError(f"unsupported splat output extension '{ext}'; expected .splat or .ply")
    raise SceneIoError("missing splat output extension; expected .splat or .ply")


def save_splats(path, scene: Scene, metadata: SplatMetadata | None = None) -> None:
    (save_splats_ply if _format(path) == "ply" else save_splats_splat)(path, scene, metadata)


def load_splats(path):
    return (load_splats_ply if _format(path) == "ply" else load_splats_splat)(path)
