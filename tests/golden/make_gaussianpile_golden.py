"""Generates tests/golden/gaussianpile_*.npz from the reference's own GaussianPile CUDA
build (oracle/_ref/gaussianplie_ref_C*.so, built by oracle/build_ref.py).

Each case stores its inputs and exactly what the reference's ProjectedSliceForwardCUDA /
ProjectedSliceBackwardCUDA return for the configuration its adapter uses (us_focus shader,
tile mapper, additive compositing). Usage on a GPU machine, from the repository root:
    python tests/golden/make_gaussianpile_golden.py [--out tests/golden]
"""

from __future__ import annotations

import argparse
import math
import sys
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]
sys.path[:0] = [str(ROOT), str(ROOT / "ultrasound-3d-reconstruction_b200"), str(ROOT / "oracle" / "_ref")]

import gaussianplie_ref_C as REF  # noqa: E402

from gaussianplie_renderer import GaussianPlieRenderConfig, build_slice_grid_pack  # noqa: E402
from gaussianplie_renderer.autograd import _meta_vector, _us_focus_params_vector  # noqa: E402
from us3d_b200 import scenes  # noqa: E402


def pose_matrix(angle_deg, axis, t):
    a = math.radians(angle_deg)
    axis = torch.tensor(axis, dtype=torch.float64)
    axis = axis / axis.norm()
    K = torch.tensor([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]], dtype=torch.float64)
    R = torch.eye(3, dtype=torch.float64) + math.sin(a) * K + (1 - math.cos(a)) * K @ K
    P = torch.eye(4, dtype=torch.float64)
    P[:3, :3] = R
    P[:3, 3] = torch.tensor(t, dtype=torch.float64)
    return P.float()


def cases():
    sc = scenes.make_scene(4000, seed=0, cube_mm=40.0, opacity_mu=-1.0)
    yield "c1", sc, pose_matrix(5.0, (1, 0.2, 0), (20.0, 1.0, 20.0)), dict(H=128, W=128, lat=0.3, ax=0.3, near=0.0,
                                                                          centre=True, sigma_z=1.0, pose_grad=True)
    sc2 = scenes.make_scene(1500, seed=1, cube_mm=30.0, log_scale_mean=0.3)
    # the pipeline passes a world->probe pose where the API expects probe->world; build the
    # probe->world pose so that its inverse still places the slice inside the cloud
    P = pose_matrix(-8.0, (0.3, 1, 0.1), (0.0, 0.0, 0.0))
    P[:3, 3] = -(P[:3, :3] @ torch.tensor([15.0, 2.0, 15.0]))
    yield "inverse_pose", sc2, torch.linalg.inv(P), dict(H=64, W=96, lat=0.4, ax=0.35, near=0.0, centre=True,
                                                         sigma_z=0.8, pose_grad=True)
    sc3 = scenes.make_scene(800, seed=3, cube_mm=24.0)
    yield "ragged", sc3, pose_matrix(12.0, (0, 0, 1), (4.0, 2.0, 12.0)), dict(H=50, W=70, lat=0.5, ax=0.45, near=2.0,
                                                                            centre=False, sigma_z=1.5, pose_grad=False)


def run(name, sc, pose, p):
    dev = torch.device("cuda")
    cfg = GaussianPlieRenderConfig(H=p["H"], W=p["W"], lateral_spacing_mm_per_pix=p["lat"],
                                   axial_spacing_mm_per_pix=p["ax"], axial_near_mm=p["near"], sigma_z_mm=p["sigma_z"])
    grid = build_slice_grid_pack(SimpleNamespace(H=p["H"], W=p["W"], delta_lateral_mm=p["lat"], delta_axial_mm=p["ax"],
                                                 near_mm=p["near"], center_lateral=p["centre"]), dev)
    meta = _meta_vector(cfg, dev)
    params = _us_focus_params_vector(cfg, dev)
    m = meta.cpu().tolist()
    G = sc.means.shape[0]
    t = [x.to(dev).float().contiguous() for x in (sc.means, sc.scales, sc.quats, sc.opacities, torch.ones(G))]
    posed = pose.to(dev).contiguous()
    colors, rects, ids, rs, re = REF.ProjectedSliceForwardCUDA(
        *t, posed, grid, params, p["H"], p["W"], m[2], m[3], m[4], int(m[5]), m[6], m[7], m[8], int(m[10]),
        int(m[11]), int(m[12]), bool(m[9]), int(m[13]), m[14], int(m[15]))
    g = torch.Generator().manual_seed(77)
    grad = torch.randn((p["H"], p["W"]), generator=g)
    dm, ds, dq, do, di, dp = REF.ProjectedSliceBackwardCUDA(
        *t, posed, grid, params, rects, 0, p["H"], p["W"], int(m[5]), m[2], m[3], m[4], m[8], int(m[13]), m[14],
        int(m[10]), ids, rs, re, grad.to(dev).reshape(-1).contiguous(), int(m[15]), bool(p["pose_grad"]))
    torch.cuda.synchronize()
    c = lambda x: x.detach().cpu().numpy()  # noqa: E731
    return dict(means=c(t[0]), scales=c(t[1]), quats=c(t[2]), opacities=c(t[3]), intensities=c(t[4]), pose=c(posed),
                grid=c(grid), params=c(params), meta=c(meta), H=p["H"], W=p["W"], pose_grad=int(p["pose_grad"]),
                grad_image=c(grad), ref_image=c(colors), ref_rects=c(rects), ref_sorted_ids=c(ids),
                ref_range_start=c(rs), ref_range_end=c(re), ref_d_means=c(dm), ref_d_scales=c(ds), ref_d_quats=c(dq),
                ref_d_opacity=c(do), ref_d_intensity=c(di), ref_d_pose=c(dp))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", type=Path, default=Path(__file__).resolve().parent)
    a = ap.parse_args()
    a.out.mkdir(parents=True, exist_ok=True)
    for name, sc, pose, p in cases():
        d = run(name, sc, pose, p)
        np.savez_compressed(a.out / f"gaussianpile_{name}.npz", **d)
        print(name, {k: v.shape for k, v in d.items() if k.startswith("ref_")})


if __name__ == "__main__":
    main()
