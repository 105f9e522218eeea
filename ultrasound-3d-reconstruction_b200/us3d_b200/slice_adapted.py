"""Host side of the slice-adapted 3DGS bounded additive splat over the C ABI."""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import torch

from . import _lib

_capacity_hint: dict = {}


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


@dataclass
class SABinning:
    workspace: torch.Tensor
    capacity: int
    total: int
    n: int
    H: int
    W: int


def bounded_forward(H, W, half_width, half_height, means2d, inv2d, weights, colors, radius_sigma=3.0,
                    capacity: Optional[int] = None):
    """(image (H*W,3), alpha (H*W,1), binning)."""
    N = int(means2d.shape[0])
    dev = means2d.device
    _lib.check(_lib.call("us3d_set_device", dev.index if dev.index is not None else torch.cuda.current_device()),
               "us3d_set_device")
    key = (N, H, W)
    cap = int(capacity if capacity is not None else _capacity_hint.get(key, max(4096, 4 * N)))
    P = H * W
    image = torch.empty((P, 3), dtype=torch.float32, device=dev)
    alpha = torch.empty((P, 1), dtype=torch.float32, device=dev)
    for _ in range(3):
        nbytes = int(_lib.call("us3d_sa_workspace_bytes", N, H, W, cap))
        ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        st = _lib.call("us3d_sa_bounded_forward", ws.data_ptr(), nbytes, N, H, W, float(half_width), float(half_height),
                       means2d.data_ptr(), inv2d.data_ptr(), weights.data_ptr(), colors.data_ptr(), float(radius_sigma),
                       cap, image.data_ptr(), alpha.data_ptr(), _stream())
        _lib.check(st, "us3d_sa_bounded_forward")
        total = ctypes.c_int64(0)
        flags = ctypes.c_int32(0)
        _lib.check(_lib.call("us3d_sa_read_status", ws.data_ptr(), ctypes.byref(total), ctypes.byref(flags),
                             _stream()), "us3d_sa_read_status")
        if flags.value == 0:
            _capacity_hint[key] = max(4096, int(total.value * 1.25) + 1024)
            return image, alpha, SABinning(ws, cap, int(total.value), N, H, W)
        cap = int(total.value * 1.25) + 1024
    raise RuntimeError("us3d_sa_bounded_forward: capacity retry failed")


def bounded_backward(b: SABinning, half_width, half_height, means2d, inv2d, weights, colors, grad_image, grad_alpha,
                     radius_sigma=3.0):
    dev = means2d.device
    N = b.n
    scratch = torch.empty(max(int(_lib.call("us3d_sa_backward_scratch_bytes", b.capacity)), 16), dtype=torch.uint8,
                          device=dev)
    dm = torch.empty((N, 2), dtype=torch.float32, device=dev)
    di = torch.empty((N, 2, 2), dtype=torch.float32, device=dev)
    dw = torch.empty((N, 1), dtype=torch.float32, device=dev)
    dc = torch.empty((N, 3), dtype=torch.float32, device=dev)
    gi = grad_image.contiguous().float()
    ga = grad_alpha.contiguous().float()
    st = _lib.call("us3d_sa_bounded_backward", b.workspace.data_ptr(), N, b.H, b.W, float(half_width),
                   float(half_height), means2d.data_ptr(), inv2d.data_ptr(), weights.data_ptr(), colors.data_ptr(),
                   gi.data_ptr(), ga.data_ptr(), float(radius_sigma), b.capacity, scratch.data_ptr(), scratch.numel(),
                   dm.data_ptr(), di.data_ptr(), dw.data_ptr(), dc.data_ptr(), _stream())
    _lib.check(st, "us3d_sa_bounded_backward")
    return dm, di, dw, dc


def export_bins(b: SABinning):
    dev = b.workspace.device
    T = ((b.W + 15) // 16) * ((b.H + 15) // 16)
    ids = torch.empty(max(b.total, 1), dtype=torch.int32, device=dev)
    rs = torch.empty(T, dtype=torch.int32, device=dev)
    re = torch.empty(T, dtype=torch.int32, device=dev)
    _lib.check(_lib.call("us3d_sa_export_bins", b.workspace.data_ptr(), b.n, b.H, b.W, b.capacity, ids.data_ptr(),
                         rs.data_ptr(), re.data_ptr(), _stream()), "us3d_sa_export_bins")
    return ids[: b.total], rs, re


def dense_forward(pixels, means2d, inv2d, weights, colors):
    P, N = int(pixels.shape[0]), int(means2d.shape[0])
    dev = pixels.device
    image = torch.zeros((P, 3), dtype=torch.float32, device=dev)
    alpha = torch.zeros((P, 1), dtype=torch.float32, device=dev)
    _lib.check(_lib.call("us3d_sa_dense_forward", P, N, pixels.data_ptr(), means2d.data_ptr(), inv2d.data_ptr(),
                         weights.data_ptr(), colors.data_ptr(), image.data_ptr(), alpha.data_ptr(), _stream()),
               "us3d_sa_dense_forward")
    return image, alpha


def dense_backward(pixels, means2d, inv2d, weights, colors, grad_image, grad_alpha):
    P, N = int(pixels.shape[0]), int(means2d.shape[0])
    dev = pixels.device
    dm = torch.zeros((N, 2), dtype=torch.float32, device=dev)
    di = torch.zeros((N, 2, 2), dtype=torch.float32, device=dev)
    dw = torch.zeros((N, 1), dtype=torch.float32, device=dev)
    dc = torch.zeros((N, 3), dtype=torch.float32, device=dev)
    gi, ga = grad_image.contiguous().float(), grad_alpha.contiguous().float()
    _lib.check(_lib.call("us3d_sa_dense_backward", P, N, pixels.data_ptr(), means2d.data_ptr(), inv2d.data_ptr(),
                         weights.data_ptr(), colors.data_ptr(), gi.data_ptr(), ga.data_ptr(), dm.data_ptr(),
                         di.data_ptr(), dw.data_ptr(), dc.data_ptr(), _stream()), "us3d_sa_dense_backward")
    return dm, di, dw, dc
