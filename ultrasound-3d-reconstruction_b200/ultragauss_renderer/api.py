"""UltraGaussRenderer with the reference's forward signature
(ops/ultragauss_renderer/ultragauss_renderer/api.py:15-55)."""

from typing import Dict, Tuple

import torch
import torch.nn as nn

from us3d_b200.lazy import LazyDict

from .autograd import _RenderFunction, lazy_pixel_csr
from .types import SliceGeometry, UltraGaussRenderConfig


class UltraGaussRenderer(nn.Module):
    def __init__(self, config: UltraGaussRenderConfig):
        super().__init__()
        self.config = config
        self.last_binning = None

    def forward(
        self,
        gauss_means_world: torch.Tensor,
        gauss_precision_tril: torch.Tensor,
        gauss_opacities: torch.Tensor,
        gauss_intensities: torch.Tensor,
        pixel_positions_world: torch.Tensor,
        geometry: SliceGeometry,
        return_intermediates: bool = False,
    ) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor, Dict[str, torch.Tensor]]:
        holder = {"want_counts": bool(return_intermediates)}
        image, alpha, depth, counts = _RenderFunction.apply(
            self.config,
            gauss_means_world,
            gauss_precision_tril,
            gauss_opacities,
            gauss_intensities,
            pixel_positions_world,
            geometry.origin_world,
            geometry.axis_lateral_world,
            geometry.axis_axial_world,
            geometry.axis_elevational_world,
            holder,
        )
        binning = holder["binning"]
        self.last_binning = binning
        cfg = self.config
        if cfg.enable_shadow:
            # Optional shadow term of the reference (api.py:37-42), applied in torch.
            delta = cfg.shadow_delta if cfg.shadow_delta > 0.0 else (1.0 / float(cfg.H))
            alpha_img = alpha.view(cfg.H, cfg.W)
            image = image.view(cfg.H, cfg.W)
            T = torch.exp(-torch.cumsum(alpha_img * delta, dim=0))
            image = (image * T).view(-1)

        image = image.view(cfg.H, cfg.W)
        alpha = alpha.view(cfg.H, cfg.W)
        depth = depth.view(cfg.H, cfg.W)
        if return_intermediates:
            off_fn, idx_fn = lazy_pixel_csr(binning, binning.pixels, counts)
            intermediates = LazyDict(
                {"pixel_gauss_offsets": off_fn, "pixel_gauss_indices": idx_fn},
                pixel_gauss_counts=counts,
            )
        else:
            intermediates = {}
        return image, alpha, depth, intermediates
