"""Autograd function over the B200 library with the reference's argument order and
gradient outputs (ops/ultragray_renderer/ultragray_renderer/autograd.py:97-262).

Per call the forward draws one uniform per ray from torch's CUDA generator, exactly as the
reference does, and turns it into an elevational ray offset with the arcsine profile; the
ray binning and the per-pixel forward state stay in the library workspace for the backward.
"""

import math

import torch

from us3d_b200 import ultragray as _ugr

from .types import UltragrayRenderConfig


def ensure_tensor(t, dtype: torch.dtype = torch.float32):
    if t is None:
        return None
    if not t.is_cuda:
        t = t.cuda()
    if t.dtype != dtype:
        t = t.to(dtype=dtype)
    return t.contiguous()


def _params(config: UltragrayRenderConfig) -> _ugr.UGRParams:
    return _ugr.UGRParams(
        width_mm=float(config.width_mm),
        near_mm=float(config.near_mm),
        lateral_col_offset=float(config.lateral_col_offset),
        elev_cutoff_mm=float(config.elev_cutoff_margin_mm),
        k_sigma=float(config.k_sigma),
        quadrature_window_radius_mm=float(config.quadrature_window_radius_mm),
        local_transmission_window_only=bool(config.local_transmission_window_only),
        local_transmission_max_window_mm=float(config.local_transmission_max_window_mm),
    )


class _UltragrayRenderFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, config, means, scales, quats, attenuations, sh_coeffs, pixel_positions, ray_origins, ray_dirs,
                probe_origin, axis_lateral, axis_elevational, axis_axial):
        means = ensure_tensor(means)
        scales = ensure_tensor(scales)
        quats = ensure_tensor(quats)
        attenuations = ensure_tensor(attenuations)
        sh_coeffs = ensure_tensor(sh_coeffs)
        pixel_positions = ensure_tensor(pixel_positions)
        ray_origins = ensure_tensor(ray_origins)
        ray_dirs = ensure_tensor(ray_dirs)
        probe_origin = ensure_tensor(probe_origin)
        axis_lateral = ensure_tensor(axis_lateral)
        axis_elevational = ensure_tensor(axis_elevational)
        axis_axial = ensure_tensor(axis_axial)

        num_rays = ray_origins.shape[0]
        u = torch.rand(num_rays, device=means.device, dtype=torch.float32)
        ray_perturbations = (torch.asin(2.0 * u - 1.0) / (math.pi / 2.0) * config.ops_max_offset_mm).contiguous()

        p = _params(config)
        image, binning = _ugr.forward(means, scales, quats, attenuations, sh_coeffs, pixel_positions, ray_origins,
                                      ray_dirs, probe_origin, axis_lateral, axis_elevational, axis_axial,
                                      ray_perturbations, p)
        ctx.params = p
        ctx.binning = binning
        ctx.save_for_backward(quats, pixel_positions, ray_origins, ray_dirs, axis_elevational, ray_perturbations)
        return image

    @staticmethod
    def backward(ctx, dL_dImage):
        quats, pixel_positions, ray_origins, ray_dirs, axis_elevational, ray_perturbations = ctx.saved_tensors
        dm, ds, dq, da, dsh = _ugr.backward(ctx.binning, quats, pixel_positions, ray_origins, ray_dirs,
                                            axis_elevational, ray_perturbations, dL_dImage.contiguous(), ctx.params)
        return (None, dm, ds, dq, da, dsh, None, None, None, None, None, None, None)
