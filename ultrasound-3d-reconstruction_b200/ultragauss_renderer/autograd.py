"""Autograd wiring of the UltraGauss renderer over the us3d_b200 C ABI.

Forward: one binning (mapper) + tile-staged shading; backward: the hand-written adjoint.
Input handling follows the reference (ops/ultragauss_renderer/ultragauss_renderer/
autograd.py:10-23): tensors are moved to CUDA, cast to fp32 and made contiguous.
"""

from __future__ import annotations

from typing import Optional

import torch

from us3d_b200 import ultragauss as _ug

from .types import UltraGaussRenderConfig


def ensure_tensor(t: Optional[torch.Tensor], dtype: torch.dtype = torch.float32) -> Optional[torch.Tensor]:
    if t is None:
        return None
    if not t.is_cuda:
        if not torch.cuda.is_available():
            raise RuntimeError("ultragauss_renderer requires CUDA: the B200 kernels are the only compute path")
        t = t.cuda()
    if t.dtype != dtype:
        t = t.to(dtype=dtype)
    return t.contiguous()


def _xyz(t: torch.Tensor) -> torch.Tensor:
    """Accepts (N,3) or the reference's padded (N,4) layout; returns contiguous (N,3)."""
    if t.dim() == 2 and t.shape[-1] == 4:
        t = t[:, :3]
    return t.contiguous()


def _spec(config: UltraGaussRenderConfig, origin, lat, ax, ele) -> _ug.SliceSpec:
    return _ug.SliceSpec(
        height=int(config.H),
        width=int(config.W),
        lateral_spacing=float(config.lateral_spacing_mm_per_pix),
        axial_spacing=float(config.axial_spacing_mm_per_pix),
        axial_near=float(config.axial_near_mm),
        lateral_col_offset=float(config.lateral_col_offset),
        origin=origin,
        axis_lat=lat,
        axis_ax=ax,
        axis_ele=ele,
    )


class _RenderFunction(torch.autograd.Function):
    """Inputs as in the reference's _RenderFunction (autograd.py:28-40) plus an optional
    ``holder`` dict that receives the binning handle; outputs are (image, alpha, depth,
    pixel_gauss_counts)."""

    @staticmethod
    def forward(ctx, config: UltraGaussRenderConfig, gauss_means_world, gauss_precision_tril, gauss_opacities,
                gauss_intensities, pixel_positions_world, probe_origin_world, axis_lateral_world,
                axis_axial_world, axis_elevational_world, holder=None):
        means_in_cols = gauss_means_world.shape[-1]
        means = _xyz(ensure_tensor(gauss_means_world))
        tril = ensure_tensor(gauss_precision_tril)
        opac = ensure_tensor(gauss_opacities).reshape(-1)
        inten = ensure_tensor(gauss_intensities).reshape(-1)
        pixels = _xyz(ensure_tensor(pixel_positions_world))
        origin = ensure_tensor(probe_origin_world)
        lat = ensure_tensor(axis_lateral_world)
        ax = ensure_tensor(axis_axial_world)
        ele = ensure_tensor(axis_elevational_world)

        n_pixels = pixels.shape[0]
        H, W = int(config.H), int(config.W)
        if n_pixels != 0 and n_pixels != H * W:
            raise RuntimeError("n_pixels must equal H*W")
        frames = _ug.build_frame_table([_spec(config, origin, lat, ax, ele)] if n_pixels else [], pixels.device)
        # Without a request for intermediates the tiles are culled to the Gaussians' in-slice
        # chi-square ellipses (identical image and gradients, no candidate counts).
        cull = holder is not None and not holder.get("want_counts", True) and n_pixels > 0
        b = _ug.bin_gaussians(means, tril, opac, inten, frames, float(config.chi2_threshold),
                              float(config.diag_beta), bool(config.mapper_sort_by_depth),
                              slice_cull_pixels=pixels if cull else None)
        image, alpha, depth, counts = _ug.forward(b, pixels, float(config.fixed_bg_alpha),
                                                  float(config.fixed_bg_intensity))
        if counts is None:
            counts = torch.zeros(0, dtype=torch.int32, device=pixels.device)
        ctx.save_for_backward(pixels, alpha)
        ctx.binning = b
        ctx.config = config
        ctx.means_cols = means_in_cols
        ctx.mark_non_differentiable(counts)
        if holder is not None:
            holder["binning"] = b
        return image, alpha, depth, counts

    @staticmethod
    def backward(ctx, d_image, d_alpha, d_depth, d_counts):
        del d_counts
        pixels, alpha = ctx.saved_tensors
        cfg = ctx.config
        dm, dt, do, di = _ug.backward(
            ctx.binning, pixels, d_image.contiguous().float(), d_alpha.contiguous().float(),
            d_depth.contiguous().float(), alpha, float(cfg.fixed_bg_alpha), float(cfg.fixed_bg_intensity),
        )
        if ctx.means_cols == 4:
            dm = torch.nn.functional.pad(dm, (0, 1))
        return None, dm, dt, do, di, None, None, None, None, None, None


def lazy_pixel_csr(binning: _ug.UGBinning, pixels: torch.Tensor, counts: torch.Tensor):
    """Thunks producing the reference's (pixel_gauss_offsets, pixel_gauss_indices)."""
    cache = {}

    def _both():
        if "v" not in cache:
            cache["v"] = _ug.pixel_csr(binning, pixels, counts)
        return cache["v"]

    return (lambda: _both()[0]), (lambda: _both()[1])
