"""Drop-in UltraGS-baseline surfel rasteriser on B200: the public names, argument order,
validation and outputs of ops/ultrags_baseline_renderer/ultrags_baseline_renderer/__init__.py
(rasterize_gaussians, GaussianRasterizationSettings, GaussianRasterizer), computed by the
us3d_b200 library. Forward returns (color (3,H,W), radii (P,), allmap (7,H,W)); backward
returns gradients in the reference's input order, including the screen-space ``means2D``
gradient it reports."""

from typing import NamedTuple

import torch
import torch.nn as nn

from us3d_b200 import surfel as _gs


def _snapshot_on_host(values):
    """Host copies of the tensors among ``values`` (detached, never aliasing device or host
    inputs), other entries passed through: what a debug-mode call saves when it fails."""
    return tuple(v.detach().to("cpu", copy=True) if torch.is_tensor(v) else v for v in values)


# the reference package exports its snapshot helper under this name
cpu_deep_copy_tuple = _snapshot_on_host


def rasterize_gaussians(means3D, means2D, sh, colors_precomp, opacities, scales, rotations, cov3Ds_precomp,
                        raster_settings):
    return _RasterizeGaussians.apply(means3D, means2D, sh, colors_precomp, opacities, scales, rotations,
                                     cov3Ds_precomp, raster_settings)


def _f32(t):
    if t is None:
        return None
    if t.numel() == 0:
        return t
    return t.to(dtype=torch.float32).contiguous()


class _RasterizeGaussians(torch.autograd.Function):
    @staticmethod
    def forward(ctx, means3D, means2D, sh, colors_precomp, opacities, scales, rotations, cov3Ds_precomp,
                raster_settings):
        s = raster_settings
        args = (s.bg, means3D, colors_precomp, opacities, scales, rotations, s.scale_modifier, cov3Ds_precomp,
                s.viewmatrix, s.projmatrix, s.tanfovx, s.tanfovy, s.image_height, s.image_width, sh, s.sh_degree,
                s.campos, s.prefiltered, s.debug)
        t = [_f32(x) if isinstance(x, torch.Tensor) else x for x in args]
        (bg, m3, cp, op, sc, rot, mod, cov, vm, pm, tfx, tfy, ih, iw, shs, deg, cam, pre, dbg) = t
        if m3.dim() != 2 or m3.shape[1] != 3:
            raise RuntimeError("means3D must have dimensions (num_points, 3)")

        def run():
            out = _gs.forward(bg, m3, cp, op.reshape(-1) if op.numel() else op, sc, rot, mod, cov, vm, pm, ih, iw,
                              shs, deg, cam, pre)
            if dbg:
                torch.cuda.synchronize()
            return out

        if s.debug:
            cpu_args = _snapshot_on_host(args)
            try:
                num_rendered, color, depth, radii, state = run()
            except Exception as ex:
                torch.save(cpu_args, "snapshot_fw.dump")
                print("\nAn error occured in forward. Please forward snapshot_fw.dump for debugging.")
                raise ex
        else:
            num_rendered, color, depth, radii, state = run()
        ctx.raster_settings = raster_settings
        ctx.num_rendered = num_rendered
        ctx.state = state
        ctx.opacity_shape = opacities.shape
        ctx.save_for_backward(cp, m3, sc, rot, cov, radii, shs)
        return color, radii, depth

    @staticmethod
    def backward(ctx, grad_out_color, grad_radii, grad_depth):
        s = ctx.raster_settings
        colors_precomp, means3D, scales, rotations, cov3Ds_precomp, radii, sh = ctx.saved_tensors
        bg, vm, pm = _f32(s.bg), _f32(s.viewmatrix), _f32(s.projmatrix)
        cam = _f32(s.campos)
        if grad_depth is None:
            grad_depth = torch.zeros((7, grad_out_color.shape[1], grad_out_color.shape[2]),
                                     dtype=torch.float32, device=grad_out_color.device)
        args = (bg, means3D, radii, colors_precomp, scales, rotations, s.scale_modifier, cov3Ds_precomp, vm, pm,
                s.tanfovx, s.tanfovy, grad_out_color, grad_depth, sh, s.sh_degree, cam, ctx.state)

        def run():
            return _gs.backward(ctx.state, bg, means3D, radii, colors_precomp, scales, rotations, s.scale_modifier,
                                cov3Ds_precomp, vm, pm, s.tanfovx, s.tanfovy, grad_out_color, grad_depth, sh,
                                s.sh_degree, cam)

        if s.debug:
            cpu_args = _snapshot_on_host(args[:-1])
            try:
                out = run()
            except Exception as ex:
                torch.save(cpu_args, "snapshot_bw.dump")
                print("\nAn error occured in backward. Writing snapshot_bw.dump for debugging.\n")
                raise ex
        else:
            out = run()
        (grad_means2D, grad_colors_precomp, grad_opacities, grad_means3D, grad_cov3Ds_precomp, grad_sh, grad_scales,
         grad_rotations) = out
        if grad_opacities.numel() == ctx.opacity_shape.numel():
            grad_opacities = grad_opacities.reshape(ctx.opacity_shape)
        return (grad_means3D, grad_means2D, grad_sh, grad_colors_precomp, grad_opacities, grad_scales,
                grad_rotations, grad_cov3Ds_precomp, None)


class GaussianRasterizationSettings(NamedTuple):
    image_height: int
    image_width: int
    tanfovx: float
    tanfovy: float
    bg: torch.Tensor
    scale_modifier: float
    viewmatrix: torch.Tensor
    projmatrix: torch.Tensor
    sh_degree: int
    campos: torch.Tensor
    prefiltered: bool
    debug: bool


class GaussianRasterizer(nn.Module):
    def __init__(self, raster_settings):
        super().__init__()
        self.raster_settings = raster_settings

    def markVisible(self, positions):
        with torch.no_grad():
            return _gs.mark_visible(positions.to(torch.float32), self.raster_settings.viewmatrix.to(torch.float32))

    def forward(self, means3D, means2D, opacities, shs=None, colors_precomp=None, scales=None, rotations=None,
                cov3D_precomp=None):
        raster_settings = self.raster_settings
        if (shs is None and colors_precomp is None) or (shs is not None and colors_precomp is not None):
            raise Exception('Please provide excatly one of either SHs or precomputed colors!')
        if ((scales is None or rotations is None) and cov3D_precomp is None) or (
                (scales is not None or rotations is not None) and cov3D_precomp is not None):
            raise Exception('Please provide exactly one of either scale/rotation pair or precomputed 3D covariance!')
        empty = torch.Tensor([]).cuda()
        shs = empty if shs is None else shs
        colors_precomp = empty if colors_precomp is None else colors_precomp
        scales = empty if scales is None else scales
        rotations = empty if rotations is None else rotations
        cov3D_precomp = empty if cov3D_precomp is None else cov3D_precomp
        return rasterize_gaussians(means3D, means2D, shs, colors_precomp, opacities, scales, rotations, cov3D_precomp,
                                   raster_settings)


__all__ = ["GaussianRasterizationSettings", "GaussianRasterizer", "rasterize_gaussians", "cpu_deep_copy_tuple"]
