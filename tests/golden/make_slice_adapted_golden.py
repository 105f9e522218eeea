"""Generates tests/golden/slice_adapted_*.npz from the reference's own slice-adapted 3DGS
CUDA build (oracle/_ref/slice_adapted_ref_C*.so and the binning harness
slice_adapted_ref_bins*.so, built by oracle/build_ref.py).

Inputs are seeded projected 2D Gaussians (the arguments of additive_splat_bounded);
outputs are what the reference's bounded_forward / bounded_backward return plus its tile
binning. Usage on a GPU machine from the repository root:
    python tests/golden/make_slice_adapted_golden.py [--out tests/golden]
"""

from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]
sys.path[:0] = [str(ROOT), str(ROOT / "ultrasound-3d-reconstruction_b200"), str(ROOT / "oracle" / "_ref")]

import slice_adapted_ref_bins as REFB  # noqa: E402
import slice_adapted_ref_C as REF  # noqa: E402


def make_inputs(N, H, W, hw, hh, seed):
    g = torch.Generator().manual_seed(seed)
    means = torch.stack([(torch.rand(N, generator=g) * 2.2 - 1.1) * hw, (torch.rand(N, generator=g) * 2.2 - 1.1) * hh], 1)
    ang = torch.rand(N, generator=g) * np.pi
    sd = torch.exp(torch.randn(N, 2, generator=g) * 0.4) * (0.015 * (hw + hh))
    c, s = torch.cos(ang), torch.sin(ang)
    R = torch.stack([torch.stack([c, -s], -1), torch.stack([s, c], -1)], -2)
    cov = R @ torch.diag_embed(sd * sd) @ R.transpose(1, 2)
    inv = torch.linalg.inv(cov)
    weights = (torch.rand(N, 1, generator=g) * 0.8 + 0.1) / torch.sqrt(torch.det(cov)).unsqueeze(1) * 0.05
    colors = torch.rand(N, 3, generator=g)
    gi = torch.randn(H * W, 3, generator=g)
    ga = 0.2 * torch.randn(H * W, 1, generator=g)
    return [x.float().contiguous() for x in (means, inv, weights, colors, gi, ga)]


def run(name, N, H, W, hw, hh, seed, rs=3.0):
    dev = torch.device("cuda")
    means, inv, weights, colors, gi, ga = [x.to(dev) for x in make_inputs(N, H, W, hw, hh, seed)]
    image, alpha = REF.bounded_forward(H, W, hw, hh, means, inv, weights, colors, rs)
    dm, di, dw, dc = REF.bounded_backward(H, W, hw, hh, means, inv, weights, colors, gi, ga, rs)
    ids, starts, ends = REFB.RefTileBinning(H, W, hw, hh, means, inv, rs)
    torch.cuda.synchronize()
    c = lambda x: x.detach().cpu().numpy()  # noqa: E731
    return dict(H=H, W=W, half_width=np.float32(hw), half_height=np.float32(hh), radius_sigma=np.float32(rs),
                means2d=c(means), inv2d=c(inv), weights=c(weights), colors=c(colors), grad_image=c(gi),
                grad_alpha=c(ga), ref_image=c(image), ref_alpha=c(alpha), ref_d_means=c(dm), ref_d_inv=c(di),
                ref_d_weights=c(dw), ref_d_colors=c(dc), ref_sorted_ids=c(ids), ref_range_start=c(starts),
                ref_range_end=c(ends))


CASES = [("small", 3000, 96, 128, 20.0, 15.0, 0), ("binned", 20000, 160, 128, 25.6, 32.0, 1),
         ("ragged", 17000, 50, 70, 12.0, 9.0, 2)]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", type=Path, default=Path(__file__).resolve().parent)
    a = ap.parse_args()
    a.out.mkdir(parents=True, exist_ok=True)
    for name, *args in CASES:
        d = run(name, *args)
        np.savez_compressed(a.out / f"slice_adapted_{name}.npz", **d)
        print(name, {k: v.shape for k, v in d.items() if k.startswith("ref_")})


if __name__ == "__main__":
    main()
