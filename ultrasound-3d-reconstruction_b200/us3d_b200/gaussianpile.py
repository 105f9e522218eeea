"""Host side of the GaussianPile projected-slice path over the C ABI."""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import torch

from . import _lib
from ._alloc import float_outputs

_capacity_hint: dict = {}


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


@dataclass
class GPBinning:
    workspace: torch.Tensor
    capacity: int
    total: int
    n_gauss: int
    H: int
    W: int
    tile: int
    k_sigma: float
    tensors: tuple  # (means, scales, quats, opac, inten, pose, grid, params) kept alive for the backward


def forward(means, scales, quats, opac, inten, pose, grid, params, H, W, lateral_spacing, axial_spacing, axial_near,
            tile_size=16, k_sigma=3.0, sort_by_v=False, capacity: Optional[int] = None):
    """Mapper + additive forward; returns (image (H,W), binning)."""
    G = int(means.shape[0])
    dev = means.device
    _lib.check(_lib.call("us3d_set_device", dev.index if dev.index is not None else torch.cuda.current_device()),
               "us3d_set_device")
    key = (G, H, W, tile_size)
    cap = int(capacity if capacity is not None else _capacity_hint.get(key, max(4096, 4 * G)))
    image = torch.empty((H, W), dtype=torch.float32, device=dev)
    args = (means, scales, quats, opac, inten, pose, grid, params)
    for _ in range(3):
        nbytes = int(_lib.call("us3d_gp_workspace_bytes", G, H, W, tile_size, cap))
        ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        st = _lib.call("us3d_gp_forward", ws.data_ptr(), nbytes, G, *(t.data_ptr() for t in args), H, W,
                       float(lateral_spacing), float(axial_spacing), float(axial_near), int(tile_size), float(k_sigma),
                       int(bool(sort_by_v)), cap, image.data_ptr(), _stream())
        _lib.check(st, "us3d_gp_forward")
        total = ctypes.c_int64(0)
        flags = ctypes.c_int32(0)
        _lib.check(_lib.call("us3d_gp_read_status", ws.data_ptr(), ctypes.byref(total), ctypes.byref(flags),
                             _stream()), "us3d_gp_read_status")
        if flags.value == 0:
            _capacity_hint[key] = max(4096, int(total.value * 1.25) + 1024)
            return image, GPBinning(ws, cap, int(total.value), G, H, W, int(tile_size), float(k_sigma), args)
        if total.value > 0x7FFFFFFF:
            raise RuntimeError(f"us3d_gp_forward: {total.value} instances exceed the int32 index range")
        cap = int(total.value * 1.25) + 1024
    raise RuntimeError("us3d_gp_forward: capacity retry failed")


GRAD_POSE = 1
GRAD_SHAPE_ANALYTIC = 2
SHAPE_GRADIENTS = ("finite_difference", "analytic")


def backward(b: GPBinning, grad_image: torch.Tensor, pose_grad: bool = False,
             shape_gradients: str = "finite_difference"):
    """(d_means, d_scales, d_quats, d_opacity, d_intensity, d_pose). ``shape_gradients``:
    "finite_difference" gives the reference's central differences (step 1e-3) for scales and
    quaternions, "analytic" their exact derivative."""
    if shape_gradients not in SHAPE_GRADIENTS:
        raise ValueError(f"shape_gradients must be one of {SHAPE_GRADIENTS}, got {shape_gradients!r}")
    flags = (GRAD_POSE if pose_grad else 0) | (GRAD_SHAPE_ANALYTIC if shape_gradients == "analytic" else 0)
    means, scales, quats, opac, inten, pose, grid, params = b.tensors
    G = b.n_gauss
    dev = means.device
    sbytes = int(_lib.call("us3d_gp_backward_scratch_bytes", G, b.capacity))
    scratch = torch.empty(max(sbytes, 16), dtype=torch.uint8, device=dev)
    # every gradient is written in full; the pose gradient only when it is asked for
    dm, ds, dq, do, di, dp = float_outputs(dev, [(G, 3), (G, 3), (G, 4), (G,), (G,), (4, 4)],
                                           zero=() if pose_grad else (5,))
    gi = grad_image.reshape(-1).contiguous().float()
    st = _lib.call("us3d_gp_backward", b.workspace.data_ptr(), G, *(t.data_ptr() for t in b.tensors), b.H, b.W, b.tile,
                   b.k_sigma, b.capacity, gi.data_ptr(), flags, scratch.data_ptr(), scratch.numel(),
                   dm.data_ptr(), ds.data_ptr(), dq.data_ptr(), do.data_ptr(), di.data_ptr(), dp.data_ptr(), _stream())
    _lib.check(st, "us3d_gp_backward")
    return dm, ds, dq, do, di, dp


def export_bins(b: GPBinning):
    """(sorted ids (I,), range_start (T,), range_end (T,), rects (G,4)) in the reference's format."""
    dev = b.workspace.device
    tx, ty = (b.W + b.tile - 1) // b.tile, (b.H + b.tile - 1) // b.tile
    ids = torch.empty(max(b.total, 1), dtype=torch.int32, device=dev)
    rs = torch.empty(tx * ty, dtype=torch.int32, device=dev)
    re = torch.empty(tx * ty, dtype=torch.int32, device=dev)
    rects = torch.empty((b.n_gauss, 4), dtype=torch.int32, device=dev)
    _lib.check(_lib.call("us3d_gp_export_bins", b.workspace.data_ptr(), b.n_gauss, b.H, b.W, b.tile, b.capacity,
                         ids.data_ptr(), rs.data_ptr(), re.data_ptr(), rects.data_ptr(), _stream()), "us3d_gp_export_bins")
    return ids[: b.total], rs, re, rects
