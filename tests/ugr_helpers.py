"""Helpers for the UltraGray tests: seeded probe scenes, fixture loading, and one B200
render + backward through the library."""

from __future__ import annotations

import math
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"

SCENE_ARRAYS = ("means", "scales", "quats", "attenuations", "sh", "pixels", "ray_o", "ray_d", "origin", "lat", "ele",
                "ax", "pert", "grad_image")
SCENE_FLOATS = ("width_mm", "near_mm", "col_off", "elev_cut", "k_sigma", "wr", "maxwin")


def make_scene(G, W, H, seed, width_mm=38.0, near_mm=2.0, depth_mm=40.0, elev_mm=2.5, scale_range=(0.25, 1.2),
               ops_max_offset_mm=0.5, wr=2.0, local=False, maxwin=17.0, k_sigma=3.0, elev_cut=0.0,
               tilted=False):
    """A linear-array probe looking down +axial with W scanlines of H samples, and G
    Gaussians spread over the imaged slab (slightly beyond it laterally and in depth)."""
    rng = np.random.default_rng(seed)
    if tilted:
        ang = 0.3
        lat = np.array([math.cos(ang), 0.0, math.sin(ang)])
        ax = np.array([-math.sin(ang), 0.0, math.cos(ang)])
        ele = np.cross(ax, lat)
        origin = np.array([1.5, -0.7, 3.0])
    else:
        lat, ele, ax = np.eye(3)
        origin = np.zeros(3)
    col_off = (W - 1) * 0.5
    spacing = width_mm / W
    xs = (np.arange(W) - col_off) * spacing
    zs = near_mm + (np.arange(H) + 0.5) * (depth_mm / H)
    ray_o = origin[None, :] + xs[:, None] * lat[None, :]
    ray_d = np.repeat(ax[None, :], W, 0)
    pixels = ray_o[:, None, :] + zs[None, :, None] * ax[None, None, :]
    u = rng.uniform(-0.55, 0.55, G) * width_mm
    v = rng.uniform(-1.0, 1.0, G) * elev_mm
    w = rng.uniform(near_mm - 2.0, near_mm + depth_mm + 2.0, G)
    means = origin[None, :] + u[:, None] * lat + v[:, None] * ele + w[:, None] * ax
    scales = np.exp(rng.uniform(np.log(scale_range[0]), np.log(scale_range[1]), (G, 3)))
    quats = rng.normal(size=(G, 4))
    quats /= np.linalg.norm(quats, axis=1, keepdims=True)
    quats *= rng.uniform(0.7, 1.4, (G, 1))  # unnormalised on purpose: the renderer normalises
    attens = rng.normal(0.5, 1.2, G)
    sh = np.concatenate([rng.uniform(0.2, 1.0, (G, 1)), rng.normal(0, 0.15, (G, 3))], 1)
    uu = rng.uniform(0, 1, W)
    pert = np.arcsin(2 * uu - 1) / (math.pi / 2) * ops_max_offset_mm
    grad_image = rng.normal(size=(H, W))
    grad_image[rng.uniform(size=(H, W)) < 0.05] = 0.0  # exercises the |dL/dB| < 1e-6 skip
    f = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
    return dict(means=f(means), scales=f(scales), quats=f(quats), attenuations=f(attens), sh=f(sh), pixels=f(pixels),
                ray_o=f(ray_o), ray_d=f(ray_d), origin=f(origin), lat=f(lat), ele=f(ele), ax=f(ax), pert=f(pert),
                grad_image=f(grad_image), width_mm=float(width_mm), near_mm=float(near_mm), col_off=float(col_off),
                elev_cut=float(elev_cut), k_sigma=float(k_sigma), wr=float(wr), local=bool(local),
                maxwin=float(maxwin))


def ugr_golden_names():
    return sorted(p.stem.split("_", 1)[1] for p in GOLDEN.glob("ultragray_*.npz"))


def load_ugr(name):
    p = GOLDEN / f"ultragray_{name}.npz"
    if not p.exists():
        import pytest

        pytest.skip(f"golden fixture {p.name} not generated")
    d = dict(np.load(p))
    scene = {k: d[k] for k in SCENE_ARRAYS}
    for k in SCENE_FLOATS:
        scene[k] = float(d[k])
    scene["local"] = bool(d["local"])
    return scene, {k: v for k, v in d.items() if k.startswith("ref_")}


def params(scene):
    from us3d_b200 import ultragray as U

    return U.UGRParams(width_mm=scene["width_mm"], near_mm=scene["near_mm"], lateral_col_offset=scene["col_off"],
                       elev_cutoff_mm=scene["elev_cut"], k_sigma=scene["k_sigma"],
                       quadrature_window_radius_mm=scene["wr"], local_transmission_window_only=scene["local"],
                       local_transmission_max_window_mm=scene["maxwin"])


def run_b200_ugr(scene, device, capacity=None, backward=True):
    import torch

    from us3d_b200 import ultragray as U

    t = {k: torch.as_tensor(scene[k]).to(device).contiguous() for k in SCENE_ARRAYS}
    p = params(scene)
    image, b = U.forward(t["means"], t["scales"], t["quats"], t["attenuations"], t["sh"], t["pixels"], t["ray_o"],
                         t["ray_d"], t["origin"], t["lat"], t["ele"], t["ax"], t["pert"], p, capacity=capacity)
    counts, offsets, idx, depths = U.export_csr(b)
    out = dict(image=image, counts=counts, offsets=offsets, indices=idx, depths=depths, total=b.total)
    if backward:
        dm, ds, dq, da, dsh = U.backward(b, t["quats"], t["pixels"], t["ray_o"], t["ray_d"], t["ele"], t["pert"],
                                         t["grad_image"], p)
        out.update(d_means=dm, d_scales=ds, d_quats=dq, d_attens=da, d_sh=dsh)
    torch.cuda.synchronize()
    return {k: (v.detach().cpu().numpy() if hasattr(v, "detach") else v) for k, v in out.items()}


def run_reference_ugr(ref, scene, device):
    """The reference's own CUDA build (MapperForwardCUDA, ShaderForwardCUDA,
    ShaderBackwardCUDA) on the scene, with means/scales padded to 4 wide as its autograd
    function does (ops/ultragray_renderer/ultragray_renderer/autograd.py:89-92, 117-118)."""
    import torch
    import torch.nn.functional as F

    t = {k: torch.as_tensor(scene[k]).to(device).contiguous() for k in SCENE_ARRAYS}
    mp = F.pad(t["means"], (0, 1)).contiguous()
    sp = F.pad(t["scales"], (0, 1)).contiguous()
    W = t["pixels"].shape[0]
    counts, offsets, idx, depths = ref.MapperForwardCUDA(mp, sp, t["origin"], t["lat"], t["ele"], t["ax"], int(W),
                                                         scene["width_mm"], scene["near_mm"], scene["col_off"],
                                                         scene["elev_cut"], scene["k_sigma"])
    args = (mp, sp, t["quats"], t["attenuations"], t["sh"], counts, offsets, idx, depths, t["pixels"], t["ray_o"],
            t["ray_d"], t["ele"], t["pert"], scene["k_sigma"], scene["wr"], bool(scene["local"]), scene["maxwin"])
    image = ref.ShaderForwardCUDA(*args)
    dm, ds, dq, da, dsh = ref.ShaderBackwardCUDA(t["grad_image"], *args)
    torch.cuda.synchronize()
    c = lambda x: x.detach().cpu().numpy()  # noqa: E731
    return dict(ref_image=c(image), ref_counts=c(counts), ref_offsets=c(offsets), ref_indices=c(idx),
                ref_depths=c(depths), ref_d_means=c(dm)[:, :3], ref_d_scales=c(ds)[:, :3], ref_d_quats=c(dq),
                ref_d_attens=c(da), ref_d_sh=c(dsh))
