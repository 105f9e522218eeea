"""GaussianPlieRenderer with the reference's interface
(ops/gaussianplie_renderer/gaussianplie_renderer/api.py:10-154)."""

import torch
import torch.nn as nn

from .autograd import render_gaussianpile_projected_slice
from .check import should_validate_inputs, validate_render_inputs
from .reference import quat_to_matrix_wxyz
from .types import GaussianPlieRenderConfig


class GaussianPlieRenderer(nn.Module):
    """GaussianPile renderer facade: Gaussians as (mean, scale, quat, alpha); the kernels
    receive an all-ones intensity."""

    def __init__(self, config: GaussianPlieRenderConfig):
        super().__init__()
        self.config = config
        self._slice_grid_geometry = None
        self._delegate = None
        # "finite_difference" (the reference's scale / quaternion gradients), "analytic" (their
        # exact derivative) or None (the process-wide default, set_shape_gradients)
        self.shape_gradients = None

    def _ensure_delegate(self):
        if self._delegate is None and self.config.backend == "ultragauss_lowmem":
            from ultragauss_renderer import UltraGaussRenderConfig, UltraGaussRenderer

            c = self.config
            self._delegate = UltraGaussRenderer(UltraGaussRenderConfig(
                H=int(c.H), W=int(c.W), lateral_spacing_mm_per_pix=float(c.lateral_spacing_mm_per_pix),
                axial_spacing_mm_per_pix=float(c.axial_spacing_mm_per_pix), axial_near_mm=float(c.axial_near_mm),
                lateral_col_offset=float(c.lateral_col_offset), chi2_threshold=float(c.radius_sigma) ** 2,
                mapper_sort_by_depth=False, fixed_bg_alpha=1.0e-6, fixed_bg_intensity=0.0, diag_beta=float(c.cov_eps),
                enable_shadow=False, shadow_delta=0.0))
        return self._delegate

    @staticmethod
    def _quat_wxyz_to_matrix(quats: torch.Tensor) -> torch.Tensor:
        return quat_to_matrix_wxyz(quats)

    def _precision_tril_from_scales_quats(self, scales: torch.Tensor, quats: torch.Tensor) -> torch.Tensor:
        """Raw lower-Cholesky precision factor (diagonal raw^2 + cov_eps) of R diag(1/s^2) R^T,
        the UltraGauss parameterisation used by the ``ultragauss_lowmem`` backend."""
        eps = float(self.config.cov_eps)
        R = quat_to_matrix_wxyz(quats)
        inv_var = 1.0 / scales.clamp_min(eps).square()
        L = torch.linalg.cholesky((R * inv_var.unsqueeze(-2)) @ R.transpose(1, 2))
        raw_diag = (torch.diagonal(L, dim1=1, dim2=2) - eps).clamp_min(1e-8).sqrt()
        return torch.stack([raw_diag[:, 0], L[:, 1, 0], L[:, 2, 0], raw_diag[:, 1], L[:, 2, 1], raw_diag[:, 2]], dim=1)

    def forward(self, gauss_means: torch.Tensor, gauss_scales: torch.Tensor, gauss_quats: torch.Tensor,
                gauss_alphas: torch.Tensor, pose_probe_to_world: torch.Tensor, pixel_positions_world: torch.Tensor = None,
                origin_world: torch.Tensor = None, axis_lateral_world: torch.Tensor = None,
                axis_axial_world: torch.Tensor = None, axis_elevational_world: torch.Tensor = None) -> torch.Tensor:
        if should_validate_inputs(self.config):
            validate_render_inputs(self.config, gauss_means, gauss_scales, gauss_quats, gauss_alphas,
                                   pose_probe_to_world)
        delegate = self._ensure_delegate()
        if self.config.backend == "ultragauss_lowmem":
            if any(t is None for t in (pixel_positions_world, origin_world, axis_lateral_world, axis_axial_world,
                                       axis_elevational_world)):
                raise RuntimeError("ultragauss_lowmem backend requires pixel positions and slice geometry axes.")
            from ultragauss_renderer import SliceGeometry

            pred, _alpha, _depth, _ = delegate(
                gauss_means_world=gauss_means,
                gauss_precision_tril=self._precision_tril_from_scales_quats(gauss_scales, gauss_quats),
                gauss_opacities=gauss_alphas, gauss_intensities=torch.ones_like(gauss_alphas),
                pixel_positions_world=pixel_positions_world,
                geometry=SliceGeometry(origin_world=origin_world, axis_lateral_world=axis_lateral_world,
                                       axis_axial_world=axis_axial_world,
                                       axis_elevational_world=axis_elevational_world),
                return_intermediates=False)
            return pred
        if self._slice_grid_geometry is None:
            raise RuntimeError("GaussianPlieRenderer requires slice_grid_geometry; call set_slice_grid_geometry().")
        return render_gaussianpile_projected_slice(self.config, gauss_means, gauss_scales, gauss_quats, gauss_alphas,
                                                   pose_probe_to_world, self._slice_grid_geometry,
                                                   shape_gradients=self.shape_gradients)

    def set_slice_grid_geometry(self, slice_grid_geometry: torch.Tensor) -> None:
        self._slice_grid_geometry = slice_grid_geometry
        if self._delegate is not None and hasattr(self._delegate, "set_slice_grid_geometry"):
            self._delegate.set_slice_grid_geometry(slice_grid_geometry)
