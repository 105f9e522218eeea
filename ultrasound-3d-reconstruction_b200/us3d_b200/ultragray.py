"""Host side of the UltraGray scanline renderer over the C ABI.

``forward`` bins the Gaussians per ray (image column) and renders the (H, W) B-mode image
in one call sequence (the reference's MapperForwardCUDA + ShaderForwardCUDA,
ops/ultragray_renderer/ultragray_renderer/autograd.py:124-178); ``backward`` reuses the
binning and the per-pixel forward state kept in the workspace
(ShaderBackwardCUDA, autograd.py:206-245).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import torch

from . import _lib

_capacity_hint: dict = {}


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _f32(t: torch.Tensor, dev) -> torch.Tensor:
    return t.to(device=dev, dtype=torch.float32).contiguous()


@dataclass
class UGRBinning:
    workspace: torch.Tensor
    capacity: int
    total: int
    n_gauss: int
    W: int
    H: int


@dataclass
class UGRParams:
    width_mm: float
    near_mm: float
    lateral_col_offset: float
    elev_cutoff_mm: float
    k_sigma: float
    quadrature_window_radius_mm: float
    local_transmission_window_only: bool
    local_transmission_max_window_mm: float


def forward(means, scales, quats, attenuations, sh_coeffs, pixel_positions, ray_origins, ray_dirs, origin,
            axis_lateral, axis_elevational, axis_axial, ray_perturbations, p: UGRParams,
            capacity: Optional[int] = None):
    """Returns (image (H, W), binning). All tensors must already be contiguous fp32 on one GPU."""
    dev = means.device
    _lib.check(_lib.call("us3d_set_device", dev.index if dev.index is not None else torch.cuda.current_device()),
               "us3d_set_device")
    G = int(means.shape[0])
    W, H = int(pixel_positions.shape[0]), int(pixel_positions.shape[1])
    key = (G, W, H)
    cap = int(capacity if capacity is not None else _capacity_hint.get(key, max(4096, 8 * G)))
    image = torch.empty((H, W), dtype=torch.float32, device=dev)
    for _ in range(3):
        nbytes = int(_lib.call("us3d_ugr_workspace_bytes", G, W, H, cap))
        ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        st = _lib.call("us3d_ugr_forward", ws.data_ptr(), nbytes, G, means.data_ptr(), scales.data_ptr(),
                       quats.data_ptr(), attenuations.data_ptr(), sh_coeffs.data_ptr(), pixel_positions.data_ptr(),
                       ray_origins.data_ptr(), ray_dirs.data_ptr(), origin.data_ptr(), axis_lateral.data_ptr(),
                       axis_elevational.data_ptr(), axis_axial.data_ptr(), ray_perturbations.data_ptr(), W, H,
                       float(p.width_mm), float(p.near_mm), float(p.lateral_col_offset), float(p.elev_cutoff_mm),
                       float(p.k_sigma), float(p.quadrature_window_radius_mm),
                       1 if p.local_transmission_window_only else 0, float(p.local_transmission_max_window_mm), cap,
                       image.data_ptr(), _stream())
        _lib.check(st, "us3d_ugr_forward")
        total = ctypes.c_int64(0)
        flags = ctypes.c_int32(0)
        _lib.check(_lib.call("us3d_ugr_read_status", ws.data_ptr(), ctypes.byref(total), ctypes.byref(flags),
                             _stream()), "us3d_ugr_read_status")
        if flags.value == 0:
            _capacity_hint[key] = max(4096, int(total.value * 1.25) + 1024)
            return image, UGRBinning(ws, cap, int(total.value), G, W, H)
        if flags.value & 2:
            raise RuntimeError("us3d_ugr_forward: per-ray and per-Gaussian instance totals disagree")
        cap = int(total.value * 1.25) + 1024
    raise RuntimeError("us3d_ugr_forward: capacity retry failed")


def backward(b: UGRBinning, quats, pixel_positions, ray_origins, ray_dirs, axis_elevational, ray_perturbations,
             grad_image, p: UGRParams):
    """Returns (d_means (G,3), d_scales (G,3), d_quats (G,4), d_attenuations (G), d_sh (G,4))."""
    dev = quats.device
    G = b.n_gauss
    scratch = torch.empty(max(int(_lib.call("us3d_ugr_backward_scratch_bytes", b.capacity)), 16), dtype=torch.uint8,
                          device=dev)
    dm = torch.empty((G, 3), dtype=torch.float32, device=dev)
    ds = torch.empty((G, 3), dtype=torch.float32, device=dev)
    dq = torch.empty((G, 4), dtype=torch.float32, device=dev)
    da = torch.empty((G,), dtype=torch.float32, device=dev)
    dsh = torch.empty((G, 4), dtype=torch.float32, device=dev)
    gi = grad_image.to(dtype=torch.float32).contiguous()
    st = _lib.call("us3d_ugr_backward", b.workspace.data_ptr(), G, quats.data_ptr(), pixel_positions.data_ptr(),
                   ray_origins.data_ptr(), ray_dirs.data_ptr(), axis_elevational.data_ptr(),
                   ray_perturbations.data_ptr(), b.W, b.H, float(p.k_sigma), float(p.quadrature_window_radius_mm),
                   1 if p.local_transmission_window_only else 0, float(p.local_transmission_max_window_mm),
                   b.capacity, gi.data_ptr(), scratch.data_ptr(), scratch.numel(), dm.data_ptr(), ds.data_ptr(),
                   dq.data_ptr(), da.data_ptr(), dsh.data_ptr(), _stream())
    _lib.check(st, "us3d_ugr_backward")
    return dm, ds, dq, da, dsh


def export_csr(b: UGRBinning):
    """(ray_counts, ray_offsets, ray_indices, sorted_depths) in MapperForwardCUDA's format."""
    dev = b.workspace.device
    counts = torch.empty(b.W, dtype=torch.int32, device=dev)
    offsets = torch.empty(b.W, dtype=torch.int32, device=dev)
    idx = torch.empty(max(b.total, 1), dtype=torch.int32, device=dev)
    depths = torch.empty(max(b.total, 1), dtype=torch.float32, device=dev)
    _lib.check(_lib.call("us3d_ugr_export_csr", b.workspace.data_ptr(), b.n_gauss, b.W, b.H, b.capacity,
                         counts.data_ptr(), offsets.data_ptr(), idx.data_ptr(), depths.data_ptr(), _stream()),
               "us3d_ugr_export_csr")
    return counts, offsets, idx[: b.total], depths[: b.total]


def ops_perturbations(num_rays: int, ops_max_offset_mm: float, device, generator=None) -> torch.Tensor:
    """Per-ray elevational offsets with the arcsine profile the reference draws
    (autograd.py:121-123): asin(2u - 1) / (pi / 2) * ops_max_offset_mm, u ~ U[0, 1)."""
    import math

    u = torch.rand(num_rays, device=device, dtype=torch.float32, generator=generator)
    return (torch.asin(2.0 * u - 1.0) / (math.pi / 2.0) * ops_max_offset_mm).contiguous()
