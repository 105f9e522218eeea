"""ctypes binding of the us3d_b200 C ABI (include/us3d_b200.h).

The library is the only compute path: if it is missing, or CUDA is unavailable, every
renderer raises instead of falling back to anything else.
"""

from __future__ import annotations

import ctypes
import os
import threading
from ctypes import c_float, c_int32, c_int64, c_size_t, c_void_p, c_char_p, POINTER

from .build import LIB_PATH

US3D_OK = 0
US3D_INVALID_ARG = 1
US3D_CAPACITY_OVERFLOW = 2
US3D_CUDA_ERROR = 3
US3D_TIMEOUT = 4

_STATUS_NAMES = {
    US3D_INVALID_ARG: "invalid argument",
    US3D_CAPACITY_OVERFLOW: "capacity overflow",
    US3D_CUDA_ERROR: "CUDA error",
    US3D_TIMEOUT: "timeout",
}


class SliceFrame(ctypes.Structure):
    """Host mirror of ``us3d_slice_frame`` (96 bytes)."""

    _fields_ = [
        ("origin", c_float * 3),
        ("axis_lat", c_float * 3),
        ("axis_ax", c_float * 3),
        ("axis_ele", c_float * 3),
        ("lateral_spacing", c_float),
        ("axial_spacing", c_float),
        ("axial_near", c_float),
        ("lateral_col_offset", c_float),
        ("height", c_int32),
        ("width", c_int32),
        ("tiles_x", c_int32),
        ("tiles_y", c_int32),
        ("pixel_offset", c_int32),
        ("tile_offset", c_int32),
        ("gauss_offset", c_int32),
        ("gauss_count", c_int32),
    ]


assert ctypes.sizeof(SliceFrame) == 96


class AdamTensor(ctypes.Structure):
    """Host mirror of ``us3d_adam_tensor`` (48 bytes)."""

    _fields_ = [
        ("param", c_void_p),
        ("grad", c_void_p),
        ("exp_avg", c_void_p),
        ("exp_avg_sq", c_void_p),
        ("numel", c_int64),
        ("activation", c_int32),
        ("reserved", c_int32),
    ]


assert ctypes.sizeof(AdamTensor) == 48
ADAM_MAX_TENSORS = 8
ADAM_IDENTITY = 0
ADAM_LOGISTIC = 1
UG_BIN_SLICE_CULL = 1
UG_BIN_LOGIT_ATTRIBUTES = 2
UG_BIN_GAUSSIAN_SETS = 4
IMAGES_F32, IMAGES_F32_DIV255, IMAGES_U8, IMAGES_U8_DIV255 = 0, 1, 2, 3

# name -> (restype, argtypes)
_SIGNATURES = {
    "us3d_last_error": (c_char_p, []),
    "us3d_version": (c_int32, []),
    "us3d_set_device": (c_int32, [c_int32]),
    "us3d_launch_count": (c_int64, []),
    "us3d_profile_stage": (c_int32, [c_char_p, c_int32]),
    "us3d_profile_collect": (c_int32, [POINTER(c_int32), POINTER(ctypes.c_double)]),
    "us3d_ug_workspace_bytes": (c_size_t, [c_int64, c_int32, c_int64, c_int64, c_int64]),
    "us3d_ug_backward_scratch_bytes": (c_size_t, [c_int64]),
    "us3d_ug_bin": (
        c_int32,
        [c_void_p, c_size_t, c_void_p, c_int32, c_int64, c_int64, c_int64, c_void_p, c_void_p, c_void_p,
         c_void_p, c_float, c_float, c_int32, c_int64, c_void_p],
    ),
    "us3d_ug_bin_ex": (
        c_int32,
        [c_void_p, c_size_t, c_void_p, c_int32, c_int64, c_int64, c_int64, c_void_p, c_void_p, c_void_p,
         c_void_p, c_float, c_float, c_int32, c_int64, c_void_p, c_int32, c_void_p],
    ),
    "us3d_ug_read_status": (c_int32, [c_void_p, POINTER(c_int64), POINTER(c_int32), c_void_p]),
    "us3d_ug_forward": (
        c_int32,
        [c_void_p, c_void_p, c_int32, c_int64, c_int64, c_int64, c_int64, c_void_p, c_float, c_float, c_float,
         c_float, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p],
    ),
    "us3d_ug_backward": (
        c_int32,
        [c_void_p, c_void_p, c_int32, c_int64, c_int64, c_int64, c_int64, c_void_p, c_void_p, c_void_p, c_void_p,
         c_void_p, c_float, c_float, c_float, c_float, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p, c_void_p,
         c_void_p],
    ),
    "us3d_ug_set_launch_config": (c_int32, [c_int32, c_int32]),
    "us3d_ug_get_launch_config": (c_int32, [POINTER(c_int32), POINTER(c_int32)]),
    "us3d_ug_set_backward_variant": (c_int32, [c_int32]),
    "us3d_ug_get_backward_variant": (c_int32, [POINTER(c_int32)]),
    "us3d_ug_set_forward_variant": (c_int32, [c_int32]),
    "us3d_ug_get_forward_variant": (c_int32, [POINTER(c_int32)]),
    "us3d_ug_refine_stats": (c_int32, [c_void_p, c_int64, c_void_p, c_void_p, c_void_p]),
    "us3d_ug_loss_scratch_bytes": (c_size_t, [c_int32]),
    "us3d_ug_loss": (
        c_int32,
        [c_void_p, c_int32, c_int64, c_void_p, c_void_p, c_float, c_float, c_void_p, c_size_t, c_void_p, c_void_p,
         c_void_p],
    ),
    "us3d_ug_backward_loss": (
        c_int32,
        [c_void_p, c_void_p, c_int32, c_int64, c_int64, c_int64, c_int64, c_void_p, c_void_p, c_void_p, c_void_p,
         c_void_p, c_float, c_float, c_float, c_float, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p, c_void_p,
         c_void_p],
    ),
    "us3d_adam_step": (
        c_int32, [POINTER(AdamTensor), c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                  c_int64, c_void_p]
    ),
    "us3d_frames_gather": (
        c_int32,
        [c_void_p, c_int64, c_void_p, c_int32, c_int32, c_int32, c_void_p, c_void_p, c_int32, c_void_p, c_void_p,
         c_void_p, c_void_p, c_void_p],
    ),
    "us3d_frames_geometry": (
        c_int32,
        [c_void_p, c_int64, c_void_p, c_int32, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
         c_void_p, c_void_p],
    ),
    "us3d_ug_pixel_csr": (
        c_int32,
        [c_void_p, c_void_p, c_int32, c_int64, c_int64, c_int64, c_int64, c_void_p, c_float, c_float, c_void_p,
         c_void_p, c_void_p],
    ),
    "us3d_ug_export_bins": (
        c_int32, [c_void_p, c_int64, c_int32, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]
    ),
    "us3d_ug_frame_instances": (
        c_int32, [c_void_p, c_int64, c_int32, c_int32, POINTER(c_int64), POINTER(c_int64), c_void_p]
    ),
    "us3d_gp_workspace_bytes": (c_size_t, [c_int64, c_int32, c_int32, c_int32, c_int64]),
    "us3d_gp_backward_scratch_bytes": (c_size_t, [c_int64, c_int64]),
    "us3d_gp_forward": (
        c_int32,
        [c_void_p, c_size_t, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
         c_void_p, c_int32, c_int32, c_float, c_float, c_float, c_int32, c_float, c_int32, c_int64, c_void_p,
         c_void_p],
    ),
    "us3d_gp_read_status": (c_int32, [c_void_p, POINTER(c_int64), POINTER(c_int32), c_void_p]),
    "us3d_gp_backward": (
        c_int32,
        [c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
         c_int32, c_int32, c_int32, c_float, c_int64, c_void_p, c_int32, c_void_p, c_size_t, c_void_p, c_void_p,
         c_void_p, c_void_p, c_void_p, c_void_p, c_void_p],
    ),
    "us3d_gp_export_bins": (
        c_int32, [c_void_p, c_int64, c_int32, c_int32, c_int32, c_int64, c_void_p, c_void_p, c_void_p, c_void_p,
                  c_void_p]
    ),
    "us3d_sa_workspace_bytes": (c_size_t, [c_int64, c_int32, c_int32, c_int64]),
    "us3d_sa_backward_scratch_bytes": (c_size_t, [c_int64]),
    "us3d_sa_bounded_forward": (
        c_int32,
        [c_void_p, c_size_t, c_int64, c_int32, c_int32, c_float, c_float, c_void_p, c_void_p, c_void_p, c_void_p,
         c_float, c_int64, c_void_p, c_void_p, c_void_p],
    ),
    "us3d_sa_read_status": (c_int32, [c_void_p, POINTER(c_int64), POINTER(c_int32), c_void_p]),
    "us3d_sa_bounded_backward": (
        c_int32,
        [c_void_p, c_int64, c_int32, c_int32, c_float, c_float, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
         c_void_p, c_float, c_int64, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p],
    ),
    "us3d_sa_export_bins": (
        c_int32, [c_void_p, c_int64, c_int32, c_int32, c_int64, c_void_p, c_void_p, c_void_p, c_void_p]
    ),
    "us3d_sa_dense_forward": (
        c_int32, [c_int64, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]
    ),
    "us3d_sa_dense_backward": (
        c_int32,
        [c_int64, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
         c_void_p, c_void_p, c_void_p],
    ),
    "us3d_sa_project_workspace_bytes": (c_size_t, [c_int64]),
    "us3d_sa_project": (
        c_int32,
        [c_void_p, c_size_t, c_int64] + [c_void_p] * 6 + [c_float] * 5 + [c_int32] + [c_void_p] * 6
        + [POINTER(c_int64), c_void_p],
    ),
    "us3d_sa_project_backward": (
        c_int32,
        [c_int64, c_int64] + [c_void_p] * 6 + [c_float] * 5 + [c_int32] + [c_void_p] * 9 + [c_void_p],
    ),
    "us3d_ugr_workspace_bytes": (c_size_t, [c_int64, c_int32, c_int32, c_int64]),
    "us3d_ugr_backward_scratch_bytes": (c_size_t, [c_int64]),
    "us3d_ugr_forward": (
        c_int32,
        [c_void_p, c_size_t, c_int64] + [c_void_p] * 13
        + [c_int32, c_int32, c_float, c_float, c_float, c_float, c_float, c_float, c_int32, c_float, c_int64,
           c_void_p, c_void_p],
    ),
    "us3d_ugr_read_status": (c_int32, [c_void_p, POINTER(c_int64), POINTER(c_int32), c_void_p]),
    "us3d_ugr_backward": (
        c_int32,
        [c_void_p, c_int64] + [c_void_p] * 6
        + [c_int32, c_int32, c_float, c_float, c_int32, c_float, c_int64, c_void_p, c_void_p, c_size_t]
        + [c_void_p] * 6,
    ),
    "us3d_ugr_export_csr": (
        c_int32, [c_void_p, c_int64, c_int32, c_int32, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]
    ),
    "us3d_gs_workspace_bytes": (c_size_t, [c_int64, c_int32, c_int32, c_int64]),
    "us3d_gs_backward_scratch_bytes": (c_size_t, [c_int64]),
    "us3d_gs_forward": (
        c_int32,
        [c_void_p, c_size_t, c_int64, c_int32, c_int32, c_void_p, c_int32, c_int32] + [c_void_p] * 5
        + [c_float] + [c_void_p] * 5 + [c_int32, c_int64, c_void_p, c_void_p, c_void_p, c_void_p],
    ),
    "us3d_gs_read_status": (c_int32, [c_void_p, POINTER(c_int64), POINTER(c_int32), c_void_p]),
    "us3d_gs_backward": (
        c_int32,
        [c_void_p, c_int64, c_int32, c_int32, c_void_p, c_int32, c_int32] + [c_void_p] * 4 + [c_float]
        + [c_void_p] * 5 + [c_float, c_float, c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_size_t]
        + [c_void_p] * 9,
    ),
    "us3d_gs_export": (
        c_int32, [c_void_p, c_int64, c_int32, c_int32, c_int64] + [c_void_p] * 7
    ),
    "us3d_gs_mark_visible": (c_int32, [c_int64, c_void_p, c_void_p, c_void_p, c_void_p]),
    "us3d_ug_render_noalloc": (
        c_int32,
        [c_void_p, c_int32, c_int64, c_int64, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_float,
         c_float, c_int32, c_float, c_float, c_void_p, c_void_p, c_void_p, c_void_p, POINTER(c_int64), c_void_p],
    ),
}

_lock = threading.Lock()
_lib = None


def exported_symbols() -> list[str]:
    return sorted(_SIGNATURES)


def load(path=None):
    """Loads (once) and returns the ctypes handle; raises if the library is absent."""
    global _lib
    with _lock:
        if _lib is not None and path is None:
            return _lib
        p = str(path or os.environ.get("US3D_B200_LIB") or LIB_PATH)
        try:
            lib = ctypes.CDLL(p)
        except OSError as exc:  # missing build: fail loudly, there is no other compute path
            raise RuntimeError(
                f"us3d_b200 CUDA library not loadable ({p}): {exc}. Build it with "
                "`python __graft_entry__.py` or us3d_b200.build.build()."
            ) from exc
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        if path is None:
            _lib = lib
        return lib


def check(status: int, what: str) -> None:
    if status == US3D_OK:
        return
    msg = load().us3d_last_error().decode("utf-8", "replace")
    kind = _STATUS_NAMES.get(status, f"status {status}")
    if status == US3D_INVALID_ARG:
        raise ValueError(f"{what}: {kind}: {msg}")
    raise RuntimeError(f"{what}: {kind}: {msg}")


def call(name: str, *args) -> int:
    return getattr(load(), name)(*args)
