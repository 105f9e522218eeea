"""Batched UltraGauss rendering: many frames of any sizes in one launch sequence.

``UltraGaussBatchRenderer(frames)(means, precision_tril, opacities, intensities, pixels)``
renders every frame of ``frames`` (a list of ``SliceSpec``) in one binning + one forward
launch and returns concatenated (image, alpha, depth) over all frames' pixels; its
backward runs one adjoint launch and returns gradients summed over the frames. This is
the batched form of the reference's per-frame UltraGaussRenderer (one frame per call).
"""

from __future__ import annotations

from typing import Optional, Sequence

import torch

from . import ultragauss as UG


class _BatchFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, frames: UG.FrameTable, params: dict, means, tril, opac, inten, pixels, holder):
        want_counts = params.get("want_counts", False)
        cull = params.get("slice_cull", True) and not want_counts
        b = UG.bin_gaussians(means, tril, opac, inten, frames, params["chi2"], params["beta"], params["sort_by_depth"],
                             capacity=params.get("capacity"), sync_check=params.get("sync_check", True),
                             slice_cull_pixels=pixels if cull else None)
        image, alpha, depth, counts = UG.forward(b, pixels, params["bg_alpha"], params["bg_intensity"],
                                                 want_counts=params.get("want_counts", False))
        ctx.b = b
        ctx.params = params
        ctx.save_for_backward(pixels, alpha)
        if holder is not None:
            holder["binning"] = b
            holder["counts"] = counts
        return image, alpha, depth

    @staticmethod
    def backward(ctx, d_image, d_alpha, d_depth):
        pixels, alpha = ctx.saved_tensors
        p = ctx.params
        dm, dt, do, di = UG.backward(ctx.b, pixels, d_image.contiguous(), d_alpha.contiguous(), d_depth.contiguous(),
                                     alpha, p["bg_alpha"], p["bg_intensity"])
        return None, None, dm, dt, do, di, None, None


class UltraGaussBatchRenderer:
    def __init__(self, frames: Sequence[UG.SliceSpec], device: torch.device, chi2_threshold: float = 7.815,
                 diag_beta: float = 1e-4, mapper_sort_by_depth: bool = True, fixed_bg_alpha: float = 1e-6,
                 fixed_bg_intensity: float = 0.0, capacity: Optional[int] = None, slice_cull: bool = True):
        self.frames = UG.build_frame_table(list(frames), device)
        self.params = dict(chi2=float(chi2_threshold), beta=float(diag_beta), sort_by_depth=bool(mapper_sort_by_depth),
                           bg_alpha=float(fixed_bg_alpha), bg_intensity=float(fixed_bg_intensity), capacity=capacity,
                           slice_cull=bool(slice_cull))
        self.last = {}

    @property
    def n_pixels(self) -> int:
        return self.frames.n_pixels

    def __call__(self, means, precision_tril, opacities, intensities, pixels):
        self.last = {}
        return _BatchFunction.apply(self.frames, self.params, means, precision_tril.contiguous(),
                                    opacities.reshape(-1), intensities.reshape(-1), pixels, self.last)
