"""Pure-PyTorch projected-slice math (the package's reference functions; same names and
meaning as ops/gaussianplie_renderer/gaussianplie_renderer/reference.py:7-114).

A Gaussian (mean, scales, rotation) is moved into the probe frame, conditioned on the
slice by an elevational Gaussian beam of width sigma_z (precision 1/sigma_z^2 added on the
elevational axis), and splatted as the 2D marginal of the conditioned Gaussian with weight
opacity * exp(-(q_c - q_e)/2) / sqrt(det Sigma_2d).
"""

from typing import Tuple

import torch
import torch.nn.functional as F


def quat_to_matrix_wxyz(quats: torch.Tensor) -> torch.Tensor:
    w, x, y, z = F.normalize(quats, dim=-1, eps=1e-8).unbind(-1)
    rows = [
        torch.stack([w * w + x * x - y * y - z * z, 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
        torch.stack([2 * (x * y + w * z), w * w - x * x + y * y - z * z, 2 * (y * z - w * x)], -1),
        torch.stack([2 * (x * z - w * y), 2 * (y * z + w * x), w * w - x * x - y * y + z * z], -1),
    ]
    return torch.stack(rows, dim=-2)


def build_covariance(scales: torch.Tensor, quats: torch.Tensor, cov_eps: float = 1.0e-6) -> torch.Tensor:
    R = quat_to_matrix_wxyz(quats)
    s2 = scales.clamp_min(float(cov_eps)).square()
    cov = (R * s2.unsqueeze(-2)) @ R.transpose(-1, -2)
    return cov + float(cov_eps) * torch.eye(3, device=scales.device, dtype=scales.dtype)


def world_to_camera(means: torch.Tensor, covariances: torch.Tensor,
                    pose_probe_to_world: torch.Tensor) -> Tuple[torch.Tensor, torch.Tensor]:
    rot_cw = pose_probe_to_world[:3, :3].transpose(0, 1)  # world -> probe rotation
    means_c = (means - pose_probe_to_world[:3, 3]) @ rot_cw.transpose(0, 1)
    covs_c = rot_cw @ covariances @ rot_cw.transpose(0, 1)
    return means_c, covs_c


def focus_project(means_c: torch.Tensor, covs_c: torch.Tensor, opacities: torch.Tensor, sigma_z: float,
                  det_eps: float = 1.0e-6, cov_eps: float = 1.0e-6) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    eye = torch.eye(3, device=means_c.device, dtype=means_c.dtype)
    prec_c = torch.linalg.inv(covs_c + float(cov_eps) * eye)
    beam = torch.zeros_like(eye)
    beam[2, 2] = 1.0 / (float(sigma_z) ** 2)
    prec_e = prec_c + beam
    covs_e = torch.linalg.inv(prec_e)
    means_e = (covs_e @ (prec_c @ means_c.unsqueeze(-1))).squeeze(-1)
    q_c = (means_c.unsqueeze(-2) @ prec_c @ means_c.unsqueeze(-1)).reshape(-1)
    q_e = (means_e.unsqueeze(-2) @ prec_e @ means_e.unsqueeze(-1)).reshape(-1)
    covs_2d = covs_e[:, :2, :2]
    det = torch.linalg.det(covs_2d).clamp_min(float(det_eps))
    alpha = opacities.reshape(-1) * torch.exp(-0.5 * (q_c - q_e)) * det.rsqrt()
    return means_e[:, :2], covs_2d, alpha


def render_reference(means: torch.Tensor, scales: torch.Tensor, quats: torch.Tensor, opacities: torch.Tensor,
                     pose_probe_to_world: torch.Tensor, xy_grid: torch.Tensor, sigma_z: float,
                     det_eps: float = 1.0e-6, cov_eps: float = 1.0e-6) -> torch.Tensor:
    covs = build_covariance(scales, quats, cov_eps=cov_eps)
    means_c, covs_c = world_to_camera(means, covs, pose_probe_to_world)
    mu2, cov2, alpha = focus_project(means_c, covs_c, opacities, sigma_z=sigma_z, det_eps=det_eps, cov_eps=cov_eps)
    prec2 = torch.linalg.inv(cov2 + float(cov_eps) * torch.eye(2, device=means.device, dtype=means.dtype))
    pts = xy_grid.reshape(-1, 2)
    out = torch.zeros(pts.shape[0], device=means.device, dtype=means.dtype)
    for g0 in range(0, mu2.shape[0], 1024):  # chunks of Gaussians bound the (G, P) temporaries
        d = pts.unsqueeze(0) - mu2[g0:g0 + 1024].unsqueeze(1)
        q = torch.einsum("gpi,gij,gpj->gp", d, prec2[g0:g0 + 1024], d)
        out = out + (alpha[g0:g0 + 1024].unsqueeze(1) * torch.exp(-0.5 * q)).sum(0)
    return out.reshape(xy_grid.shape[:-1])
