"""ctypes binding of libgsr.so (include/gsr.h).

The library is the product: every render, sort, scan, loss and optimizer call
goes through it. Loading fails loudly if the shared object is missing or was
built for another architecture; there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgsr.so")

GSR_OK = 0
GSR_ERR_INVALID_ARG = 1
STATUS_NAMES = {
    0: "GSR_OK",
    1: "GSR_ERR_INVALID_ARG",
    2: "GSR_ERR_OOM",
    3: "GSR_ERR_CAPACITY",
    4: "GSR_ERR_CUDA",
    5: "GSR_ERR_TIMEOUT",
    6: "GSR_ERR_NOT_READY",
}

GSR_SH_F32 = 0
GSR_SH_BF16 = 1
GSR_ADJOINT_EXACT = 0
GSR_ADJOINT_REFERENCE = 1
GSR_SCHEDULE_DEFAULT = 0
GSR_SCHEDULE_PERSISTENT = 1
GSR_SCHEDULE_GRID = 2


class gsr_config(C.Structure):
    _fields_ = [
        ("cov_blur", C.c_float),
        ("background", C.c_float * 3),
        ("tile_w", C.c_uint32),
        ("tile_h", C.c_uint32),
        ("batch", C.c_uint32),
        ("sh_dtype", C.c_int32),
        ("adjoint", C.c_int32),
        ("deterministic", C.c_int32),
        ("fp64_conic", C.c_int32),
        ("max_splats", C.c_uint64),
        ("max_views", C.c_uint32),
        ("schedule", C.c_uint32),
        ("max_pixels", C.c_uint64),
        ("max_isects", C.c_uint64),
    ]


class gsr_camera(C.Structure):
    _fields_ = [
        ("viewmat", C.c_float * 16),
        ("fx", C.c_float),
        ("fy", C.c_float),
        ("cx", C.c_float),
        ("cy", C.c_float),
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("campos", C.c_float * 3),
        ("_pad", C.c_float),
    ]


class gsr_splats(C.Structure):
    _fields_ = [
        ("transforms", C.c_void_p),
        ("sh", C.c_void_p),
        ("raw_opacity", C.c_void_p),
        ("n", C.c_uint32),
        ("sh_degree", C.c_uint32),
    ]


class gsr_grads(C.Structure):
    _fields_ = [("v_transforms", C.c_void_p), ("v_sh", C.c_void_p), ("v_raw_opacity", C.c_void_p)]


class gsr_adam_state(C.Structure):
    _fields_ = [
        ("m_transforms", C.c_void_p),
        ("v_transforms", C.c_void_p),
        ("m_sh", C.c_void_p),
        ("v_sh", C.c_void_p),
        ("m_opacity", C.c_void_p),
        ("v_opacity", C.c_void_p),
    ]


class gsr_lr(C.Structure):
    _fields_ = [
        ("position", C.c_float),
        ("rotation", C.c_float),
        ("scale", C.c_float),
        ("color", C.c_float),
        ("opacity", C.c_float),
        ("beta1", C.c_float),
        ("beta2", C.c_float),
        ("eps", C.c_float),
    ]


class gsr_train_params(C.Structure):
    _fields_ = [
        ("lr", gsr_lr),
        ("step", C.c_int32),
        ("l1_weight", C.c_float),
        ("ssim_weight", C.c_float),
        ("use_visible", C.c_int32),
    ]


GSR_TOPO_EXISTING, GSR_TOPO_REFINE_EXISTING, GSR_TOPO_REFINE_NEW = 0, 1, 2


class gsr_topo_row(C.Structure):
    _fields_ = [("source", C.c_uint32), ("kind", C.c_int32), ("sample_scalar", C.c_float), ("_pad", C.c_uint32)]


class gsr_topo_params(C.Structure):
    _fields_ = [("has_refine_decay", C.c_int32), ("scale_decay", C.c_float), ("opacity_decay", C.c_float),
                ("train_t", C.c_float), ("opacity_reset", C.c_int32), ("opacity_reset_cap", C.c_float)]


class gsr_frame(C.Structure):
    _fields_ = [("offset", C.c_uint64), ("width", C.c_uint32), ("height", C.c_uint32)]


GSR_TUNE_CANDIDATES = 9


class gsr_tune_candidate(C.Structure):
    _fields_ = [("tile_w", C.c_uint32), ("tile_h", C.c_uint32), ("batch", C.c_uint32), ("status", C.c_int32),
                ("ms_per_view", C.c_float), ("_pad", C.c_uint32)]


class gsr_tune_result(C.Structure):
    _fields_ = [("tile_w", C.c_uint32), ("tile_h", C.c_uint32), ("batch", C.c_uint32), ("ms_per_view", C.c_float),
                ("candidates", gsr_tune_candidate * GSR_TUNE_CANDIDATES)]


EXPORTED = [
    "gsr_create",
    "gsr_destroy",
    "gsr_last_error",
    "gsr_version",
    "gsr_sync_status",
    "gsr_reserve_isects",
    "gsr_prefix_sum_u32",
    "gsr_prefix_sum_u32_noalloc",
    "gsr_radix_sort_by_key_u32",
    "gsr_render_forward",
    "gsr_render_backward",
    "gsr_export",
    "gsr_loss",
    "gsr_frames_to_targets",
    "gsr_adam_step",
    "gsr_accumulate_densify",
    "gsr_train_step",
    "gsr_train_step_after",
    "gsr_profile",
    "gsr_profile_read",
    "gsr_graph_kernel_count",
    "gsr_autotune",
    "gsr_topology_apply",
    "gsr_selftest_wait_timeout",
]

PROFILE_STAGES = ("project", "depth_sort", "offsets", "emit", "tile_sort", "ranges", "raster_fwd", "visible", "loss",
                  "raster_bwd", "reduce", "project_bwd", "adam")

_lib = None


class GsrError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def load():
    """Load libgsr.so and declare its prototypes (raises if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libgsr.so not found at {LIB_PATH}; build it with `make -C rustscan_b200/csrc`")
    L = C.CDLL(LIB_PATH)
    vp, u32, i32, f32 = C.c_void_p, C.c_uint32, C.c_int32, C.c_float
    L.gsr_create.argtypes = [C.POINTER(gsr_config), C.POINTER(C.c_void_p)]
    L.gsr_destroy.argtypes = [vp]
    L.gsr_destroy.restype = None
    L.gsr_last_error.argtypes = [vp]
    L.gsr_last_error.restype = C.c_char_p
    L.gsr_version.restype = C.c_char_p
    L.gsr_sync_status.argtypes = [vp, vp, C.POINTER(C.c_uint64)]
    L.gsr_reserve_isects.argtypes = [vp, C.c_uint64]
    L.gsr_prefix_sum_u32.argtypes = [vp, vp, vp, u32, vp]
    L.gsr_prefix_sum_u32_noalloc.argtypes = [vp, vp, u32, vp]
    L.gsr_radix_sort_by_key_u32.argtypes = [vp, vp, vp, vp, vp, u32, vp]
    L.gsr_render_forward.argtypes = [vp, C.POINTER(gsr_splats), C.POINTER(gsr_camera), u32, vp, vp, vp]
    L.gsr_render_backward.argtypes = [vp, C.POINTER(gsr_splats), vp, C.POINTER(gsr_grads), vp, vp]
    L.gsr_export.argtypes = [vp, u32, i32, vp, C.c_uint64, vp]
    L.gsr_loss.argtypes = [vp, vp, vp, C.POINTER(gsr_camera), u32, f32, f32, vp, vp, vp]
    L.gsr_frames_to_targets.argtypes = [vp, vp, C.POINTER(gsr_frame), C.POINTER(gsr_camera), u32, vp, vp]
    L.gsr_adam_step.argtypes = [vp, vp, vp, vp, u32, u32, C.POINTER(gsr_grads), C.POINTER(gsr_adam_state),
                                C.POINTER(gsr_lr), i32, vp]
    L.gsr_accumulate_densify.argtypes = [vp, C.POINTER(gsr_grads), vp, vp, u32, u32, i32, vp, vp]
    L.gsr_train_step.argtypes = [vp, vp, vp, vp, u32, u32, C.POINTER(gsr_adam_state), C.POINTER(gsr_camera), u32,
                                 vp, C.POINTER(gsr_train_params), vp, vp, i32, vp]
    L.gsr_train_step_after.argtypes = [vp, vp, vp, vp, u32, u32, C.POINTER(gsr_adam_state), C.POINTER(gsr_camera),
                                       u32, vp, C.POINTER(gsr_train_params), vp, vp, i32, vp, vp]
    L.gsr_profile.argtypes = [vp, i32]
    L.gsr_profile_read.argtypes = [vp, C.POINTER(C.c_float), i32, vp]
    L.gsr_graph_kernel_count.argtypes = [vp]
    L.gsr_topology_apply.argtypes = [vp, C.POINTER(gsr_splats), vp, u32, C.POINTER(gsr_topo_params), vp, vp, vp, vp]
    L.gsr_selftest_wait_timeout.argtypes = [vp, u32, vp]
    L.gsr_autotune.argtypes = [C.POINTER(gsr_config), C.POINTER(gsr_splats), C.POINTER(gsr_camera), u32, i32,
                               C.POINTER(gsr_tune_result), vp]
    for name in EXPORTED:
        if name not in ("gsr_destroy", "gsr_last_error", "gsr_version"):
            getattr(L, name).restype = C.c_int
    _lib = L
    return L
