"""Host side of the UltraGS-baseline surfel rasteriser over the C ABI.

``forward`` replaces RasterizeGaussiansCUDA and ``backward`` RasterizeGaussiansBackwardCUDA
(ops/ultrags_baseline_renderer/rasterize_points.cu:41-233); the per-call state the
reference keeps in its geometry / binning / image byte buffers lives in one workspace here.
"""

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


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    """NULL for an absent or empty tensor (the reference passes empty tensors for absent
    inputs and tests their data pointers)."""
    if t is None or t.numel() == 0:
        return None
    return t.data_ptr()


@dataclass
class GSState:
    workspace: torch.Tensor
    capacity: int
    total: int
    P: int
    W: int
    H: int


def forward(background, means3D, colors, opacity, scales, rotations, scale_modifier, transmat_precomp, viewmatrix,
            projmatrix, image_height, image_width, sh, degree, campos, prefiltered,
            capacity: Optional[int] = None):
    """Returns (num_rendered, color (3,H,W), others (7,H,W), radii (P,), state)."""
    dev = means3D.device
    _lib.check(_lib.call("us3d_set_device", dev.index if dev.index is not None else torch.cuda.current_device()),
               "us3d_set_device")
    P = int(means3D.shape[0])
    H, W = int(image_height), int(image_width)
    M = int(sh.shape[1]) if (sh is not None and sh.numel() > 0 and sh.dim() >= 2) else 0
    if P == 0:
        return (0, torch.zeros((3, H, W), dtype=torch.float32, device=dev),
                torch.zeros((7, H, W), dtype=torch.float32, device=dev), torch.zeros((0,), dtype=torch.int32, device=dev),
                None)
    # a call that returns has written every pixel of both images (the shading kernel covers
    # all tiles) and every radius (the preprocess writes one per Gaussian)
    color = torch.empty((3, H, W), dtype=torch.float32, device=dev)
    others = torch.empty((7, H, W), dtype=torch.float32, device=dev)
    radii = torch.empty((P,), dtype=torch.int32, device=dev)
    key = (P, W, H)
    cap = int(capacity if capacity is not None else _capacity_hint.get(key, max(4096, 4 * P)))
    for _ in range(3):
        nbytes = int(_lib.call("us3d_gs_workspace_bytes", P, W, H, cap))
        ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        st = _lib.call("us3d_gs_forward", ws.data_ptr(), nbytes, P, int(degree), M, background.data_ptr(), W, H,
                       means3D.data_ptr(), _ptr(sh), _ptr(colors), opacity.data_ptr(), _ptr(scales),
                       float(scale_modifier), _ptr(rotations), _ptr(transmat_precomp), viewmatrix.data_ptr(),
                       projmatrix.data_ptr(), _ptr(campos), 1 if prefiltered else 0, cap, color.data_ptr(),
                       others.data_ptr(), radii.data_ptr(), _stream())
        _lib.check(st, "us3d_gs_forward")
        total = ctypes.c_int64(0)
        flags = ctypes.c_int32(0)
        _lib.check(_lib.call("us3d_gs_read_status", ws.data_ptr(), ctypes.byref(total), ctypes.byref(flags),
                             _stream()), "us3d_gs_read_status")
        if flags.value & 4:
            raise RuntimeError("Point is filtered although prefiltered is set. This shouldn't happen!")
        if flags.value & 2:
            raise RuntimeError("us3d_gs_forward: per-tile and per-Gaussian instance totals disagree")
        if flags.value == 0:
            _capacity_hint[key] = max(4096, int(total.value * 1.25) + 1024)
            return int(total.value), color, others, radii, GSState(ws, cap, int(total.value), P, W, H)
        cap = int(total.value * 1.25) + 1024
    raise RuntimeError("us3d_gs_forward: capacity retry failed")


def backward(state: Optional[GSState], background, means3D, radii, colors, scales, rotations, scale_modifier,
             transmat_precomp, viewmatrix, projmatrix, tan_fovx, tan_fovy, dL_dout_color, dL_dout_others, sh, degree,
             campos):
    """Returns (dmeans2D, dcolors, dopacity, dmeans3D, dtransMat, dsh, dscales, drotations) with
    the reference's shapes ((P,3), (P,3), (P,1), (P,3), (P,9), (P,M,3), (P,2), (P,4))."""
    dev = means3D.device
    P = int(means3D.shape[0])
    M = int(sh.shape[1]) if (sh is not None and sh.numel() > 0 and sh.dim() >= 2) else 0
    z = lambda *s: torch.zeros(s, dtype=torch.float32, device=dev)  # noqa: E731
    if P == 0 or state is None:
        return z(P, 3), z(P, 3), z(P, 1), z(P, 3), z(P, 9), z(P, M, 3), z(P, 2), z(P, 4)
    # the backward writes every entry of each gradient it is given; the others stay zero
    has_sh, has_sc, has_rot = M > 0 and _ptr(sh) is not None, _ptr(scales) is not None, _ptr(rotations) is not None
    dmeans2D, dcolors, dopacity, dmeans3D, dtrans, dsh, dscales, drot = float_outputs(
        dev, [(P, 3), (P, 3), (P, 1), (P, 3), (P, 9), (P, M, 3), (P, 2), (P, 4)],
        zero=[i for i, given in ((5, has_sh), (6, has_sc), (7, has_rot)) if not given])
    H, W = int(dL_dout_color.shape[1]), int(dL_dout_color.shape[2])
    scratch = torch.empty(max(int(_lib.call("us3d_gs_backward_scratch_bytes", state.capacity)), 16),
                          dtype=torch.uint8, device=dev)
    gc = dL_dout_color.to(dtype=torch.float32).contiguous()
    go = dL_dout_others.to(dtype=torch.float32).contiguous()
    st = _lib.call("us3d_gs_backward", state.workspace.data_ptr(), P, int(degree), M, background.data_ptr(), W, H,
                   means3D.data_ptr(), _ptr(sh), _ptr(colors), _ptr(scales), float(scale_modifier), _ptr(rotations),
                   _ptr(transmat_precomp), viewmatrix.data_ptr(), projmatrix.data_ptr(), _ptr(campos),
                   float(tan_fovx), float(tan_fovy), radii.data_ptr(), state.capacity, gc.data_ptr(), go.data_ptr(),
                   scratch.data_ptr(), scratch.numel(), dmeans2D.data_ptr(), dcolors.data_ptr(), dopacity.data_ptr(),
                   dmeans3D.data_ptr(), dtrans.data_ptr(), dsh.data_ptr() if has_sh else None,
                   dscales.data_ptr() if has_sc else None, drot.data_ptr() if has_rot else None,
                   _stream())
    _lib.check(st, "us3d_gs_backward")
    return dmeans2D, dcolors, dopacity, dmeans3D, dtrans, dsh, dscales, drot


def export(state: GSState):
    """(point_list, keys, ranges (T,2), n_contrib (2,H,W), accum (3,H,W), records (P,20))."""
    dev = state.workspace.device
    T = ((state.W + 15) // 16) * ((state.H + 15) // 16)
    n = max(state.total, 1)
    pl = torch.empty(n, dtype=torch.int32, device=dev)
    keys = torch.empty(n, dtype=torch.int64, device=dev)
    ranges = torch.empty((T, 2), dtype=torch.int32, device=dev)
    nc = torch.empty((2, state.H, state.W), dtype=torch.int32, device=dev)
    acc = torch.empty((3, state.H, state.W), dtype=torch.float32, device=dev)
    rec = torch.empty((max(state.P, 1), 20), dtype=torch.float32, device=dev)
    _lib.check(_lib.call("us3d_gs_export", state.workspace.data_ptr(), state.P, state.W, state.H, state.capacity,
                         pl.data_ptr(), keys.data_ptr(), ranges.data_ptr(), nc.data_ptr(), acc.data_ptr(),
                         rec.data_ptr(), _stream()), "us3d_gs_export")
    return pl[: state.total], keys[: state.total], ranges, nc, acc, rec[: state.P]


def mark_visible(means3D, viewmatrix):
    P = int(means3D.shape[0])
    out = torch.zeros(P, dtype=torch.uint8, device=means3D.device)
    _lib.check(_lib.call("us3d_gs_mark_visible", P, means3D.contiguous().data_ptr(),
                         viewmatrix.contiguous().data_ptr(), out.data_ptr(), _stream()), "us3d_gs_mark_visible")
    return out.bool()
