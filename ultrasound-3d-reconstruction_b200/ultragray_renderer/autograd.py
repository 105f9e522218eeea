"""Autograd function over the B200 library with the reference's argument order and
gradient outputs (ops/ultragray_renderer/ultragray_renderer/autograd.py:97-262).

Per call the forward draws one uniform per ray from torch's CUDA generator, exactly as the
reference does, and turns it into an elevational ray offset with the arcsine profile; the
ray binning and the per-pixel forward state stay in the library workspace for the backward.

Opt-in profiling, as the reference's (autograd.py:13-70, 149-188, 258-266): with
ULTRAGRAY_PROFILE_EVERY=n (> 0) every n-th call after the first ULTRAGRAY_PROFILE_WARMUP calls
prints one ``[ULTRAGRAY_PROFILE]`` line for its forward (wall and CUDA-event time of the
binning + shading launch sequence, which this library runs as one call, and the per-ray hit
statistics: total, active rays, mean, p50/p90/p99, max) and one for its backward.
"""

import math
import os
import time

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


_PROFILE_STEP = 0


def _env_int(name: str) -> int:
    try:
        return int(os.environ.get(name, "0"))
    except ValueError:
        return 0


def _should_profile(step: int) -> bool:
    every = _env_int("ULTRAGRAY_PROFILE_EVERY")
    return every > 0 and step > _env_int("ULTRAGRAY_PROFILE_WARMUP") and step % every == 0


def _timed(fn):
    """(result, wall ms, CUDA-event ms) of fn on the current stream, synchronised on both sides."""
    torch.cuda.synchronize()
    st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    st.record()
    out = fn()
    en.record()
    torch.cuda.synchronize()
    return out, (time.perf_counter() - t0) * 1e3, st.elapsed_time(en)


def ray_stats(ray_counts: torch.Tensor, total_hits: int) -> str:
    """Hit statistics of a ray list: total, active rays, mean over all and over active rays,
    p50 / p90 / p99 over active rays (torch.quantile, linear), max."""
    counts = ray_counts.float()
    n = ray_counts.numel()
    act = counts[ray_counts > 0]
    if act.numel():
        q = torch.quantile(act, torch.tensor([0.5, 0.9, 0.99], device=act.device)).tolist()
        mean_act = float(act.mean())
    else:
        q, mean_act = [0.0, 0.0, 0.0], 0.0
    return (f"total_hits={int(total_hits)} active_rays={int(act.numel())}/{n} "
            f"hits_mean_all={float(counts.mean()) if n else 0.0:.1f} hits_mean_active={mean_act:.1f} "
            f"hits_p50={q[0]:.1f} hits_p90={q[1]:.1f} hits_p99={q[2]:.1f} "
            f"hits_max={int(ray_counts.max()) if n else 0}")


class _UltragrayRenderFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, config, means, scales, quats, attenuations, sh_coeffs, pixel_positions, ray_origins, ray_dirs,
                probe_origin, axis_lateral, axis_elevational, axis_axial):
        global _PROFILE_STEP
        _PROFILE_STEP += 1
        ctx.profile_step = _PROFILE_STEP
        ctx.profile_enabled = _should_profile(_PROFILE_STEP)
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

        def run_forward():
            return _ugr.forward(means, scales, quats, attenuations, sh_coeffs, pixel_positions, ray_origins, ray_dirs,
                                probe_origin, axis_lateral, axis_elevational, axis_axial, ray_perturbations, p)

        if ctx.profile_enabled:
            (image, binning), wall_ms, gpu_ms = _timed(run_forward)
            counts = _ugr.export_csr(binning)[0]
            print(f"[ULTRAGRAY_PROFILE] step={ctx.profile_step} phase=forward "
                  f"mapper_shader_fwd_wall_ms={wall_ms:.3f} mapper_shader_fwd_gpu_ms={gpu_ms:.3f} "
                  f"{ray_stats(counts, binning.total)}", flush=True)
        else:
            image, binning = run_forward()
        ctx.params = p
        ctx.binning = binning
        ctx.save_for_backward(quats, pixel_positions, ray_origins, ray_dirs, axis_elevational, ray_perturbations)
        return image

    @staticmethod
    def backward(ctx, dL_dImage):
        quats, pixel_positions, ray_origins, ray_dirs, axis_elevational, ray_perturbations = ctx.saved_tensors

        def run_backward():
            return _ugr.backward(ctx.binning, quats, pixel_positions, ray_origins, ray_dirs, axis_elevational,
                                 ray_perturbations, dL_dImage.contiguous(), ctx.params)

        if ctx.profile_enabled:
            (dm, ds, dq, da, dsh), wall_ms, gpu_ms = _timed(run_backward)
            print(f"[ULTRAGRAY_PROFILE] step={ctx.profile_step} phase=backward "
                  f"shader_bwd_wall_ms={wall_ms:.3f} shader_bwd_gpu_ms={gpu_ms:.3f}", flush=True)
        else:
            dm, ds, dq, da, dsh = run_backward()
        return (None, dm, ds, dq, da, dsh, None, None, None, None, None, None, None)
