"""Generates tests/golden/slice_projection_*.npz: the slice-adapted adapter's projection of
3D Gaussians (baselines/slice_adapted_3dgs/render.py:66-98) and its PyTorch autograd
vector-Jacobian product, computed by importing the reference adapter module in this
container (its projection is plain PyTorch and runs on the CPU in float32).

The reference module's own helpers do the view transform and the camera-space covariances
(_view_points, _camera_covariances); the few lines of the adapter's function body that
follow them (slice sigma, cull, 2x2 inverse, weights) are restated below, since they are not
callable on their own. Usage from the repository root, where the reference tree is present:
    python tests/golden/make_slice_projection_golden.py [--reference /path/to/reference]
"""

from __future__ import annotations

import argparse
import os
import importlib.util
import math
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent

CASES = {
    # name: (G, seed, settings)
    "default": (4000, 0, dict(slice_thickness_mm=0.3, cull_std=3.0, thickness_scale=1.0, min_covariance=1e-4,
                              normalize_by_footprint=True)),
    "thick_nonorm": (3000, 1, dict(slice_thickness_mm=1.2, cull_std=2.0, thickness_scale=1.5, min_covariance=1e-3,
                                   normalize_by_footprint=False)),
}


def load_adapter(reference: Path):
    spec = importlib.util.spec_from_file_location("ref_slice_adapter",
                                                  reference / "baselines" / "slice_adapted_3dgs" / "render.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def make_inputs(G, seed):
    g = torch.Generator().manual_seed(seed)
    ang = 0.4
    view = torch.eye(4)
    c, s = math.cos(ang), math.sin(ang)
    view[:3, :3] = torch.tensor([[c, 0.0, s], [0.0, 1.0, 0.0], [-s, 0.0, c]])
    view[3, :3] = torch.tensor([0.7, -1.1, 0.4])  # row-vector convention: translation in the last row
    means = (torch.rand(G, 3, generator=g) - 0.5) * torch.tensor([30.0, 24.0, 8.0]) + torch.tensor([0.0, 0.0, 10.0])
    scales = torch.exp(torch.randn(G, 3, generator=g) * 0.5) * 0.4
    quats = torch.randn(G, 4, generator=g)
    quats[:5] = torch.tensor([1e-12, 0.0, 0.0, 0.0])  # below the normalisation epsilon
    opac = torch.rand(G, generator=g)
    colors = torch.rand(G, 3, generator=g)
    return [x.float().contiguous() for x in (means, scales, quats, opac, colors, view)]


def run(adapter, G, seed, st, focal_depth=10.0):
    means, scales, quats, opac, colors, view = make_inputs(G, seed)
    leaves = [x.clone().requires_grad_(True) for x in (means, scales, quats, opac, colors)]
    m, sc, q, o, col = leaves
    dtype, device = m.dtype, m.device
    means_cam = adapter._view_points(m, view)
    rel_z = means_cam[:, 2] - float(focal_depth)
    cov_cam = adapter._camera_covariances(sc, q, view)
    min_cov = float(st["min_covariance"])
    cov2d = cov_cam[:, :2, :2] + torch.eye(2, dtype=dtype, device=device).unsqueeze(0) * min_cov
    var_z = torch.clamp(cov_cam[:, 2, 2], min=min_cov)
    sigma_z = torch.sqrt(var_z + float(st["slice_thickness_mm"]) ** 2)
    keep = torch.abs(rel_z) <= float(st["cull_std"]) * sigma_z * float(st["thickness_scale"])
    means2d = means_cam[keep, :2]
    cov2d = cov2d[keep]
    rel_z = rel_z[keep]
    sigma_z = sigma_z[keep]
    colors_k = col[keep].to(dtype=dtype)
    opac_k = o.reshape(-1, 1)[keep].to(dtype=dtype)
    det = torch.clamp(cov2d[:, 0, 0] * cov2d[:, 1, 1] - cov2d[:, 0, 1] * cov2d[:, 1, 0], min=min_cov)
    inv = torch.stack([torch.stack([cov2d[:, 1, 1] / det, -cov2d[:, 0, 1] / det], -1),
                       torch.stack([-cov2d[:, 1, 0] / det, cov2d[:, 0, 0] / det], -1)], -2)
    weights = opac_k * torch.exp(-0.5 * (rel_z / torch.clamp(sigma_z, min=1.0e-6)).square()).unsqueeze(-1)
    if st["normalize_by_footprint"]:
        weights = weights / torch.sqrt(det).unsqueeze(-1)
    gen = torch.Generator().manual_seed(seed + 100)
    N = int(keep.sum())
    ups = [torch.randn(N, 2, generator=gen), torch.randn(N, 2, 2, generator=gen), torch.randn(N, 1, generator=gen),
           torch.randn(N, 3, generator=gen)]
    loss = sum((a * b).sum() for a, b in zip((means2d, inv, weights, colors_k), ups))
    loss.backward()
    n = lambda t: t.detach().numpy()  # noqa: E731
    out = dict(means=n(means), scales=n(scales), quats=n(quats), opacities=n(opac), colors=n(colors), view=n(view),
               focal_depth=np.float32(focal_depth), up_means2d=n(ups[0]), up_inv2d=n(ups[1]), up_weights=n(ups[2]),
               up_colors=n(ups[3]), ref_keep=n(keep), ref_means2d=n(means2d), ref_inv2d=n(inv),
               ref_weights=n(weights), ref_colors=n(colors_k))
    for k, leaf in zip(("means", "scales", "quats", "opacities", "colors"), leaves):
        out["ref_d_" + k] = n(leaf.grad)
    for k, v in st.items():
        out["set_" + k] = np.float32(v) if not isinstance(v, bool) else np.bool_(v)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=Path, default=os.environ.get("US3D_REFERENCE"),
                    required=not os.environ.get("US3D_REFERENCE"),
                    help="reference checkout (default: $US3D_REFERENCE)")
    ap.add_argument("--out", type=Path, default=HERE)
    a = ap.parse_args()
    adapter = load_adapter(a.reference)
    for name, (G, seed, st) in CASES.items():
        d = run(adapter, G, seed, st)
        np.savez_compressed(a.out / f"slice_projection_{name}.npz", **d)
        print(name, int(d["ref_keep"].sum()), "kept of", G)


if __name__ == "__main__":
    main()
