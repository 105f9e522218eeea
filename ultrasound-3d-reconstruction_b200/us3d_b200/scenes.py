"""Seeded synthetic scenes and probe sweeps (the real ultrasound datasets are not available
offline; these stand in with the distributions the workloads are specified by).

Headline scene: G anisotropic Gaussians in a 64 mm cube, means uniform, per-axis
log-scales N(log 1.0 mm, 0.3), uniformly random unit quaternions, intensity U(0,1),
opacity sigmoid(N(0,1)). Frames: planar B-mode slices from a linear sweep (probe moved
along the elevational axis, tilt N(0, 2 deg) about the lateral axis). All draws come from
one ``torch.Generator`` in a fixed order.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List

import torch


@dataclass
class GaussianScene:
    means: torch.Tensor  # (G,3)
    scales: torch.Tensor  # (G,3)
    quats: torch.Tensor  # (G,4) wxyz, unit
    opacities: torch.Tensor  # (G,)
    intensities: torch.Tensor  # (G,)
    precision_tril: torch.Tensor  # (G,6) raw factor, l11,l12,l13,l22,l23,l33

    def to(self, device) -> "GaussianScene":
        return GaussianScene(*(getattr(self, f).to(device) for f in
                               ("means", "scales", "quats", "opacities", "intensities", "precision_tril")))


@dataclass
class Slice:
    height: int
    width: int
    lateral_spacing: float
    axial_spacing: float
    axial_near: float
    lateral_col_offset: float
    origin: torch.Tensor
    axis_lat: torch.Tensor
    axis_ax: torch.Tensor
    axis_ele: torch.Tensor
    pixels: torch.Tensor  # (H*W, 3) world positions of pixel centres

    def to(self, device) -> "Slice":
        return Slice(self.height, self.width, self.lateral_spacing, self.axial_spacing, self.axial_near,
                     self.lateral_col_offset, *(getattr(self, f).to(device) for f in
                                                ("origin", "axis_lat", "axis_ax", "axis_ele", "pixels")))


def quat_to_rot(q: torch.Tensor) -> torch.Tensor:
    """Rotation matrices of unit (w,x,y,z) quaternions."""
    w, x, y, z = q.unbind(-1)
    return torch.stack(
        [
            1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
            2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
            2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y),
        ],
        dim=-1,
    ).reshape(*q.shape[:-1], 3, 3)


def precision_tril_from_scales_quats(scales: torch.Tensor, quats: torch.Tensor, beta: float = 1e-4) -> torch.Tensor:
    """Raw lower-Cholesky factor of Lambda = R diag(1/s^2) R^T with diagonal raw^2 + beta
    (the parameterisation UltraGauss learns); computed in float64 with elementwise operations
    only, written out for 3x3 matrices: batched BLAS / LAPACK kernels may round differently
    from run to run (buffer alignment, threads), which would make the scenes, and results that
    sit on a threshold, differ between processes."""
    s = scales.double().clamp_min(beta)
    R = quat_to_rot(quats.double())
    inv = 1.0 / (s * s)

    def lam(i, j):  # Lambda_ij = sum_k R_ik R_jk / s_k^2
        return (R[:, i, 0] * R[:, j, 0] * inv[:, 0] + R[:, i, 1] * R[:, j, 1] * inv[:, 1]
                + R[:, i, 2] * R[:, j, 2] * inv[:, 2])

    a00, a10, a20, a11, a21, a22 = lam(0, 0), lam(1, 0), lam(2, 0), lam(1, 1), lam(2, 1), lam(2, 2)
    l00 = a00.sqrt()
    l10 = a10 / l00
    l20 = a20 / l00
    l11 = (a11 - l10 * l10).sqrt()
    l21 = (a21 - l20 * l10) / l11
    l22 = (a22 - l20 * l20 - l21 * l21).sqrt()

    def raw(d):
        return (d - beta).clamp_min(1e-8).sqrt()

    return torch.stack([raw(l00), l10, l20, raw(l11), l21, raw(l22)], dim=1).float()


def make_scene(n: int, seed: int = 0, cube_mm: float = 64.0, log_scale_mean: float = 0.0,
               log_scale_std: float = 0.3, opacity_mu: float = 0.0, opacity_std: float = 1.0,
               beta: float = 1e-4) -> GaussianScene:
    # The transcendental functions and the quaternion norm run in float64 on elementwise
    # operations and are rounded to float32 once: CPU kernels evaluate exp / sigmoid / norms with
    # vector and scalar code paths whose last bits differ, and which elements take which path can
    # change from process to process.
    g = torch.Generator().manual_seed(seed)
    means = torch.rand((n, 3), generator=g) * cube_mm
    scales64 = torch.exp(log_scale_mean + log_scale_std * torch.randn((n, 3), generator=g).double())
    q = torch.randn((n, 4), generator=g).double()
    q = q / (q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1] + q[:, 2] * q[:, 2] + q[:, 3] * q[:, 3]).sqrt().clamp_min(1e-12)[:, None]
    intensities = torch.rand((n,), generator=g)
    opacities = torch.sigmoid(opacity_mu + opacity_std * torch.randn((n,), generator=g).double()).float()
    tril = precision_tril_from_scales_quats(scales64, q, beta)
    return GaussianScene(means, scales64.float(), q.float(), opacities, intensities, tril)


def slice_pixels(origin, lat, ax, H, W, lateral_spacing, axial_spacing, axial_near, col_offset) -> torch.Tensor:
    """Pixel-centre world positions, row-major (row = axial), as the reference pipeline
    builds them (pipeline_god_file.py:299-306)."""
    u = torch.arange(W, dtype=torch.float32)
    v = torch.arange(H, dtype=torch.float32)
    lateral_mm = (u - col_offset) * lateral_spacing
    axial_mm = axial_near + v * axial_spacing
    yy, xx = torch.meshgrid(axial_mm, lateral_mm, indexing="ij")
    pix = origin.view(1, 1, 3) + xx[..., None] * lat.view(1, 1, 3) + yy[..., None] * ax.view(1, 1, 3)
    return pix.reshape(-1, 3).contiguous()


def _rot_about(axis: torch.Tensor, angle: float) -> torch.Tensor:
    axis = axis / axis.norm()
    x, y, z = axis.tolist()
    c, s = math.cos(angle), math.sin(angle)
    C = 1 - c
    return torch.tensor([[c + x * x * C, x * y * C - z * s, x * z * C + y * s],
                         [y * x * C + z * s, c + y * y * C, y * z * C - x * s],
                         [z * x * C - y * s, z * y * C + x * s, c + z * z * C]], dtype=torch.float32)


def linear_sweep(n_frames: int, H: int, W: int, spacing_mm: float, seed: int = 0, cube_mm: float = 64.0,
                 step_mm: float = 2.0, tilt_deg: float = 2.0) -> List[Slice]:
    """Probe translated ``step_mm`` per frame along elevation through the cube centre,
    each frame tilted about its lateral axis by N(0, tilt_deg)."""
    g = torch.Generator().manual_seed(seed + 1_000_003)
    tilts = torch.randn((n_frames,), generator=g) * math.radians(tilt_deg)
    out = []
    col_off = (W - 1) * 0.5
    depth_mm = H * spacing_mm
    for f in range(n_frames):
        z = cube_mm * 0.5 + (f - (n_frames - 1) * 0.5) * step_mm
        lat0 = torch.tensor([1.0, 0.0, 0.0])
        ax0 = torch.tensor([0.0, 1.0, 0.0])
        ele0 = torch.tensor([0.0, 0.0, 1.0])
        R = _rot_about(lat0, float(tilts[f]))
        ax = R @ ax0
        ele = R @ ele0
        centre = torch.tensor([cube_mm * 0.5, cube_mm * 0.5, z])
        origin = centre - ax * (depth_mm * 0.5)
        pix = slice_pixels(origin, lat0, ax, H, W, spacing_mm, spacing_mm, 0.0, col_off)
        out.append(Slice(H, W, spacing_mm, spacing_mm, 0.0, col_off, origin, lat0.clone(), ax, ele, pix))
    return out
