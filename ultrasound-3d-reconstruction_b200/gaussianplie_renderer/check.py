"""Optional input validation (reference ops/gaussianplie_renderer/gaussianplie_renderer/check.py:6-29)."""

import torch

from .types import GaussianPlieRenderConfig


def should_validate_inputs(config: GaussianPlieRenderConfig) -> bool:
    return bool(config.enable_input_checks)


def validate_render_inputs(config: GaussianPlieRenderConfig, gauss_means: torch.Tensor, gauss_scales: torch.Tensor,
                           gauss_quats: torch.Tensor, gauss_opacities: torch.Tensor,
                           pose_probe_to_world: torch.Tensor) -> None:
    del config
    n = gauss_means.shape[0]
    checks = (
        (gauss_means.ndim == 2 and tuple(gauss_means.shape) == (n, 3), "gauss_means must be (N, 3)", gauss_means),
        (tuple(gauss_scales.shape) == (n, 3), "gauss_scales must be (N, 3)", gauss_scales),
        (tuple(gauss_quats.shape) == (n, 4), "gauss_quats must be (N, 4)", gauss_quats),
        (tuple(gauss_opacities.shape) in ((n,), (n, 1)), "gauss_opacities must be (N,) or (N, 1)", gauss_opacities),
        (tuple(pose_probe_to_world.shape) == (4, 4), "pose_probe_to_world must be (4, 4)", pose_probe_to_world),
    )
    for ok, msg, t in checks:
        if not ok:
            raise ValueError(f"{msg}, got {tuple(t.shape)}.")
