"""The slice-adapted 3DGS frame render with the projection fused on the GPU.

``render_slice_adapted_3dgs(gaussians, camera, settings)`` has the signature, inputs and
outputs of the reference adapter baselines/slice_adapted_3dgs/render.py:60-129 (any objects
with the fields of its dataclasses are accepted; the same dataclasses are defined here).
The reference projects the 3D Gaussians with about thirty PyTorch operations and boolean-mask
gathers; here one library call projects, culls and compacts them in index order and one
computes the projection's vector-Jacobian product, around the bounded splat. Gradients reach
means, scales_3d, quats, opacities and colors (not the view transform).
"""

from dataclasses import dataclass, field
from typing import Dict, Optional

import torch

from us3d_b200 import slice_adapted as _sa

from .api import additive_splat_bounded


@dataclass
class SliceCameraInput:
    image_height: int
    image_width: int
    half_width_mm: float
    half_height_mm: float
    focal_depth_mm: float
    world_view_transform: torch.Tensor


@dataclass
class SliceAdapted3DGSInput:
    means: torch.Tensor
    scales_3d: torch.Tensor
    quats: torch.Tensor
    opacities: torch.Tensor
    colors: torch.Tensor


@dataclass
class SliceAdaptedRenderSettings:
    slice_thickness_mm: float = 0.3
    cull_std: float = 3.0
    thickness_scale: float = 1.0
    min_covariance: float = 1.0e-4
    normalize_by_footprint: bool = True
    clamp_output: bool = True
    bg_color: float = 0.0
    output_grayscale: bool = True


@dataclass
class RenderOutput:
    image: torch.Tensor
    depth: Optional[torch.Tensor] = None
    extras: Dict[str, torch.Tensor] = field(default_factory=dict)


class _SliceProject(torch.autograd.Function):
    @staticmethod
    def forward(ctx, means, scales, quats, opacities, colors, view, settings):
        c = lambda t: t.detach().to(dtype=torch.float32).contiguous()  # noqa: E731
        m, s, q, o, col, v = c(means), c(scales), c(quats), c(opacities).reshape(-1), c(colors), c(view)
        m2, inv, w, colk, idx, mask = _sa.project(m, s, q, o, col, v, settings)
        ctx.settings = settings
        ctx.opacity_shape = opacities.shape
        ctx.save_for_backward(m, s, q, o, v, idx)
        ctx.mark_non_differentiable(mask)
        return m2, inv, w, colk, mask

    @staticmethod
    def backward(ctx, d_m2, d_inv, d_w, d_col, _d_mask):
        m, s, q, o, v, idx = ctx.saved_tensors
        n = idx.shape[0]
        z = lambda g, *sh: torch.zeros(sh, device=m.device) if g is None else g  # noqa: E731
        dm, ds, dq, dop, dc = _sa.project_backward(idx, m, s, q, o, v, ctx.settings, z(d_m2, n, 2), z(d_inv, n, 2, 2),
                                                   z(d_w, n, 1), z(d_col, n, 3))
        return dm, ds, dq, dop.reshape(ctx.opacity_shape), dc, None, None


def _finalize(image, alpha, keep, settings):
    if settings.output_grayscale:
        image = (0.299 * image[0] + 0.587 * image[1] + 0.114 * image[2]).unsqueeze(0)
    return RenderOutput(image=image, depth=None, extras={"visibility_filter": keep, "alpha_image": alpha})


def render_slice_adapted_3dgs(gaussians, camera, settings) -> RenderOutput:
    device = gaussians.means.device
    if device.type != "cuda" or gaussians.means.dtype != torch.float32:
        raise RuntimeError("This simplified delivery renderer expects CUDA float32 tensors for additive_splat_bounded.")
    view = camera.world_view_transform.to(device=device, dtype=gaussians.means.dtype)
    ps = _sa.ProjectionSettings(focal_depth=float(camera.focal_depth_mm),
                                slice_thickness=float(settings.slice_thickness_mm), cull_std=float(settings.cull_std),
                                thickness_scale=float(settings.thickness_scale),
                                min_covariance=float(settings.min_covariance),
                                normalize_by_footprint=bool(settings.normalize_by_footprint))
    means2d, inv, weights, colors, keep = _SliceProject.apply(gaussians.means, gaussians.scales_3d, gaussians.quats,
                                                              gaussians.opacities, gaussians.colors, view, ps)
    H, W = int(camera.image_height), int(camera.image_width)
    if means2d.shape[0] == 0:
        image = torch.full((3, H, W), float(settings.bg_color), device=device, dtype=gaussians.means.dtype)
        return _finalize(image, None, keep, settings)
    image_flat, alpha_flat = additive_splat_bounded(H, W, float(camera.half_width_mm), float(camera.half_height_mm),
                                                    means2d, inv, weights, colors, float(settings.cull_std))
    image_flat = image_flat + float(settings.bg_color)
    if settings.clamp_output:
        image_flat = image_flat.clamp(0.0, 1.0)
    image = image_flat.transpose(0, 1).reshape(3, H, W)
    alpha = alpha_flat.transpose(0, 1).reshape(1, H, W)
    return _finalize(image, alpha, keep, settings)
