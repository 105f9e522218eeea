"""Additive 2D Gaussian splatting with the reference's interface
(ops/slice_adapted_3dgs_renderer/slice_adapted_3dgs_renderer/api.py:1-303)."""

import torch

from us3d_b200 import slice_adapted as _sa


def _check_inputs(pixels, means2d, inv2d, weights, colors) -> None:
    if not pixels.is_cuda:
        raise ValueError("pixels must be CUDA tensors")
    tensors = [means2d, inv2d, weights, colors]
    if any(not t.is_cuda for t in tensors):
        raise ValueError("all additive_splat inputs must be CUDA tensors")
    if pixels.dtype != torch.float32 or any(t.dtype != torch.float32 for t in tensors):
        raise ValueError("additive_splat currently supports float32 only")
    if pixels.dim() != 2 or pixels.shape[-1] != 2:
        raise ValueError(f"pixels must have shape (P, 2), got {tuple(pixels.shape)}")
    _check_shapes(means2d, inv2d, weights, colors)


def _check_shapes(means2d, inv2d, weights, colors) -> None:
    if means2d.dim() != 2 or means2d.shape[-1] != 2:
        raise ValueError(f"means2d must have shape (N, 2), got {tuple(means2d.shape)}")
    n = means2d.shape[0]
    if inv2d.shape != (n, 2, 2):
        raise ValueError(f"inv2d must have shape (N, 2, 2), got {tuple(inv2d.shape)}")
    if weights.shape != (n, 1):
        raise ValueError(f"weights must have shape (N, 1), got {tuple(weights.shape)}")
    if colors.shape != (n, 3):
        raise ValueError(f"colors must have shape (N, 3), got {tuple(colors.shape)}")


def _check_bounded_inputs(image_height, image_width, half_width, half_height, means2d, inv2d, weights, colors,
                          radius_sigma) -> None:
    if image_height <= 0 or image_width <= 0:
        raise ValueError("image dimensions must be positive")
    if half_width <= 0.0 or half_height <= 0.0:
        raise ValueError("physical half extents must be positive")
    if radius_sigma <= 0.0:
        raise ValueError("radius_sigma must be positive")
    tensors = [means2d, inv2d, weights, colors]
    if any(not t.is_cuda for t in tensors):
        raise ValueError("all additive_splat_bounded inputs must be CUDA tensors")
    if any(t.dtype != torch.float32 for t in tensors):
        raise ValueError("additive_splat_bounded currently supports float32 only")
    _check_shapes(means2d, inv2d, weights, colors)


class _AdditiveSplat(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pixels, means2d, inv2d, weights, colors):
        _check_inputs(pixels, means2d, inv2d, weights, colors)
        t = [x.contiguous() for x in (pixels, means2d, inv2d, weights, colors)]
        image, alpha = _sa.dense_forward(*t)
        ctx.save_for_backward(*t)
        return image, alpha

    @staticmethod
    def backward(ctx, grad_image, grad_alpha):
        pixels, means2d, inv2d, weights, colors = ctx.saved_tensors
        gm, gi, gw, gc = _sa.dense_backward(pixels, means2d, inv2d, weights, colors, grad_image, grad_alpha)
        return None, gm, gi, gw, gc


class _AdditiveSplatBounded(torch.autograd.Function):
    @staticmethod
    def forward(ctx, image_height, image_width, half_width, half_height, means2d, inv2d, weights, colors,
                radius_sigma):
        _check_bounded_inputs(image_height, image_width, half_width, half_height, means2d, inv2d, weights, colors,
                              radius_sigma)
        t = [x.contiguous() for x in (means2d, inv2d, weights, colors)]
        image, alpha, b = _sa.bounded_forward(int(image_height), int(image_width), float(half_width),
                                              float(half_height), *t, float(radius_sigma))
        ctx.b = b
        ctx.geom = (float(half_width), float(half_height), float(radius_sigma))
        ctx.save_for_backward(*t)
        return image, alpha

    @staticmethod
    def backward(ctx, grad_image, grad_alpha):
        means2d, inv2d, weights, colors = ctx.saved_tensors
        hw, hh, rs = ctx.geom
        gm, gi, gw, gc = _sa.bounded_backward(ctx.b, hw, hh, means2d, inv2d, weights, colors, grad_image, grad_alpha,
                                              rs)
        return None, None, None, None, gm, gi, gw, gc, None


def additive_splat(pixels: torch.Tensor, means2d: torch.Tensor, inv2d: torch.Tensor, weights: torch.Tensor,
                   colors: torch.Tensor):
    """Additively splat 2D Gaussians onto flattened pixels (P, 2) in physical slice units.

    Returns image (P, 3) and alpha (P, 1).
    """
    return _AdditiveSplat.apply(pixels, means2d, inv2d, weights, colors)


def additive_splat_bounded(image_height: int, image_width: int, half_width: float, half_height: float,
                           means2d: torch.Tensor, inv2d: torch.Tensor, weights: torch.Tensor, colors: torch.Tensor,
                           radius_sigma: float = 3.0):
    """Additively splat 2D Gaussians onto an H x W image using bounded footprints.

    Returns image (H*W, 3) and alpha (H*W, 1).
    """
    return _AdditiveSplatBounded.apply(int(image_height), int(image_width), float(half_width), float(half_height),
                                       means2d, inv2d, weights, colors, float(radius_sigma))
