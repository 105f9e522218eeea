"""Autograd wiring of the GaussianPile projected-slice renderer over the us3d_b200 C ABI.

The meta and us_focus parameter vectors are built with the values the reference sends
to its kernels (ops/gaussianplie_renderer/gaussianplie_renderer/autograd.py:16-55): the
us_focus shader with a fixed elevational PSF sigma_z, det_gamma 0.5, weight threshold
max(opacity_cull_threshold, 1e-12), the tile mapper, additive compositing and no depth
ordering inside a tile.
"""

from __future__ import annotations

import torch

from us3d_b200 import gaussianpile as _gp

from .types import GaussianPlieRenderConfig

_META_LEN = 16
_US_FOCUS_PARAMS_LEN = 14

SHADER_WEIGHT_US_FOCUS = 2


def _meta_vector(config: GaussianPlieRenderConfig, device: torch.device) -> torch.Tensor:
    sz = float(config.sigma_z_mm)
    vals = [0.0] * _META_LEN
    vals[0], vals[1] = float(config.H), float(config.W)
    vals[2], vals[3] = float(config.lateral_spacing_mm_per_pix), float(config.axial_spacing_mm_per_pix)
    vals[4] = float(config.axial_near_mm)
    vals[5] = float(config.tile_size_px)
    vals[6] = max(float(config.radius_sigma) * sz, sz * 0.5)  # elevational corridor half-width (unused by us_focus)
    vals[8] = float(config.radius_sigma)
    vals[11] = vals[12] = 5.0
    vals[15] = float(SHADER_WEIGHT_US_FOCUS)
    return torch.tensor(vals, dtype=torch.float32, device=device)


def _us_focus_params_vector(config: GaussianPlieRenderConfig, device: torch.device) -> torch.Tensor:
    sz = float(config.sigma_z_mm)
    vals = [0.0] * _US_FOCUS_PARAMS_LEN
    vals[0], vals[2], vals[3] = sz, sz, sz  # sigma_ele = clamp(sz + 0 * depth, sz, sz)
    vals[4], vals[6], vals[7] = 1.0, 0.5, 8.0  # lateral focus parameters (lateral focus off)
    vals[8] = 0.5  # det_gamma
    vals[9] = float(config.det_eps)
    vals[10] = max(float(config.opacity_cull_threshold), 1.0e-12)
    return torch.tensor(vals, dtype=torch.float32, device=device)


# How scale and quaternion gradients are formed: "finite_difference" is the reference's
# central difference (step 1e-3) of the footprint/adjoint dot product; "analytic" is its exact
# derivative (no counterpart in the reference), which a caller optimising shapes may prefer.
SHAPE_GRADIENTS = _gp.SHAPE_GRADIENTS
_default_shape_gradients = "finite_difference"


def set_shape_gradients(mode: str) -> None:
    """Process-wide default for renderers whose ``shape_gradients`` attribute is None."""
    global _default_shape_gradients
    if mode not in SHAPE_GRADIENTS:
        raise ValueError(f"shape_gradients must be one of {SHAPE_GRADIENTS}, got {mode!r}")
    _default_shape_gradients = mode


def get_shape_gradients() -> str:
    return _default_shape_gradients


class _GaussianPileProjectedSliceCudaFunction(torch.autograd.Function):
    """Same inputs as the reference function of this name (autograd.py:58-137), plus an
    optional tenth: the shape-gradient mode (default: the process-wide setting)."""

    @staticmethod
    def forward(ctx, gauss_means, gauss_scales, gauss_quats, gauss_opacities, gauss_intensities,
                pose_probe_to_world, slice_grid_geometry, meta, us_focus_params, shape_gradients=None):
        ctx.shape_gradients = shape_gradients or _default_shape_gradients
        if not gauss_means.is_cuda:
            raise RuntimeError("gaussianplie_renderer requires CUDA tensors: the B200 kernels are the only compute path")
        dev = gauss_means.device
        f = lambda t: t.to(device=dev, dtype=torch.float32).contiguous()  # noqa: E731
        means, scales, quats = f(gauss_means), f(gauss_scales), f(gauss_quats)
        opac, inten = f(gauss_opacities).reshape(-1), f(gauss_intensities).reshape(-1)
        pose = f(pose_probe_to_world).reshape(16).contiguous()
        grid = f(slice_grid_geometry).reshape(-1)
        params = f(us_focus_params).reshape(-1)
        m = meta.detach().cpu().tolist()  # one host read, as the reference's .item() calls
        H, W = int(m[0]), int(m[1])
        if grid.numel() < 16:  # the reference builds a default linear, centred pack
            grid = torch.tensor([0.0, H, W, m[2], m[3], m[4], (W - 1) * 0.5, 1.0] + [0.0] * 8, dtype=torch.float32,
                                device=dev)
        image, b = _gp.forward(means, scales, quats, opac, inten, pose, grid, params, H, W, float(m[2]), float(m[3]),
                               float(m[4]), int(m[5]), float(m[8]), bool(m[9] != 0.0))
        ctx.b = b
        ctx.pose_dtype = pose_probe_to_world.dtype
        ctx.dtypes = (gauss_means.dtype, gauss_scales.dtype, gauss_quats.dtype, gauss_opacities.dtype,
                      gauss_intensities.dtype)
        ctx.shapes = (gauss_opacities.shape, gauss_intensities.shape)
        ctx.aux_shapes = (slice_grid_geometry, meta, us_focus_params)
        return image

    @staticmethod
    def backward(ctx, grad_colors_hw):
        b = ctx.b
        if grad_colors_hw is None:
            grad_colors_hw = torch.zeros((b.H, b.W), device=b.workspace.device)
        dm, ds, dq, do, di, dp = _gp.backward(b, grad_colors_hw, bool(ctx.needs_input_grad[5]),
                                              shape_gradients=ctx.shape_gradients)
        grid, meta, params = ctx.aux_shapes
        md, sd, qd, od, idt = ctx.dtypes
        grads = (dm.to(md), ds.to(sd), dq.to(qd), do.reshape(ctx.shapes[0]).to(od), di.reshape(ctx.shapes[1]).to(idt),
                 dp.to(ctx.pose_dtype), torch.zeros_like(grid), torch.zeros_like(meta), torch.zeros_like(params))
        # one gradient per input given to apply (nine, or ten with the mode)
        return (grads + (None,))[:len(ctx.needs_input_grad)]


def render_gaussianpile_projected_slice(config: GaussianPlieRenderConfig, gauss_means: torch.Tensor,
                                        gauss_scales: torch.Tensor, gauss_quats: torch.Tensor,
                                        gauss_alphas: torch.Tensor, pose_probe_to_world: torch.Tensor,
                                        slice_grid_geometry: torch.Tensor, shape_gradients=None) -> torch.Tensor:
    """(H, W) additive image; intensities are fixed to one, as in the reference
    (autograd.py:218-246). ``shape_gradients`` ("finite_difference" / "analytic", None: the
    process-wide default) chooses how the backward forms scale and quaternion gradients."""
    if not gauss_means.is_cuda:
        raise RuntimeError("GaussianPile requires CUDA tensors; the B200 kernels are the only compute path.")
    device = gauss_means.device
    return _GaussianPileProjectedSliceCudaFunction.apply(
        gauss_means, gauss_scales, gauss_quats, gauss_alphas, torch.ones_like(gauss_alphas), pose_probe_to_world,
        slice_grid_geometry.to(device=device, dtype=torch.float32), _meta_vector(config, device),
        _us_focus_params_vector(config, device), shape_gradients)
