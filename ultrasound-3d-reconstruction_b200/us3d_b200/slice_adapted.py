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


@dataclass
class ProjectionSettings:
    focal_depth: float
    slice_thickness: float
    cull_std: float
    thickness_scale: float
    min_covariance: float
    normalize_by_footprint: bool


def project(means, scales, quats, opacities, colors, viewmatrix, s: ProjectionSettings):
    """Fused slice projection. Returns (means2d (N,2), inv2d (N,2,2), weights (N,1),
    colors (N,3), keep_idx (N,), keep_mask (G,)) for the N kept Gaussians, in index order."""
    G = int(means.shape[0])
    dev = means.device
    _lib.check(_lib.call("us3d_set_device", dev.index if dev.index is not None else torch.cuda.current_device()),
               "us3d_set_device")
    nbytes = int(_lib.call("us3d_sa_project_workspace_bytes", G))
    ws = torch.empty(max(nbytes, 16), dtype=torch.uint8, device=dev)
    m2 = torch.empty((G, 2), dtype=torch.float32, device=dev)
    inv = torch.empty((G, 2, 2), dtype=torch.float32, device=dev)
    w = torch.empty((G, 1), dtype=torch.float32, device=dev)
    col = torch.empty((G, 3), dtype=torch.float32, device=dev)
    idx = torch.empty((G,), dtype=torch.int32, device=dev)
    mask = torch.zeros((G,), dtype=torch.uint8, device=dev)
    kept = ctypes.c_int64(0)
    _lib.check(_lib.call("us3d_sa_project", ws.data_ptr(), ws.numel(), G, means.data_ptr(), scales.data_ptr(),
                         quats.data_ptr(), opacities.data_ptr(), colors.data_ptr(), viewmatrix.data_ptr(),
                         float(s.focal_depth), float(s.slice_thickness), float(s.cull_std), float(s.thickness_scale),
                         float(s.min_covariance), 1 if s.normalize_by_footprint else 0, m2.data_ptr(), inv.data_ptr(),
                         w.data_ptr(), col.data_ptr(), idx.data_ptr(), mask.data_ptr(), ctypes.byref(kept),
                         _stream()), "us3d_sa_project")
    n = int(kept.value)
    return m2[:n], inv[:n], w[:n], col[:n], idx[:n], mask.bool()


def project_backward(keep_idx, means, scales, quats, opacities, viewmatrix, s: ProjectionSettings, d_means2d,
                     d_inv2d, d_weights, d_colors_kept):
    G, N = int(means.shape[0]), int(keep_idx.shape[0])
    dev = means.device
    z = lambda *sh: torch.empty(sh, dtype=torch.float32, device=dev)  # noqa: E731
    dm, ds, dq, dop, dc = z(G, 3), z(G, 3), z(G, 4), z(G), z(G, 3)
    c = lambda t: t.to(dtype=torch.float32).contiguous()  # noqa: E731
    g = [c(d_means2d), c(d_inv2d), c(d_weights), c(d_colors_kept)]
    _lib.check(_lib.call("us3d_sa_project_backward", G, N, keep_idx.data_ptr(), means.data_ptr(), scales.data_ptr(),
                         quats.data_ptr(), opacities.data_ptr(), viewmatrix.data_ptr(), float(s.focal_depth),
                         float(s.slice_thickness), float(s.cull_std), float(s.thickness_scale),
                         float(s.min_covariance), 1 if s.normalize_by_footprint else 0, g[0].data_ptr(),
                         g[1].data_ptr(), g[2].data_ptr(), g[3].data_ptr(), dm.data_ptr(), ds.data_ptr(),
                         dq.data_ptr(), dop.data_ptr(), dc.data_ptr(), _stream()), "us3d_sa_project_backward")
    return dm, ds, dq, dop, dc
