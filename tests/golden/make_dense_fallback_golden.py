"""Generates tests/golden/dense_fallback_small.npz by importing the reference's training script
(pipeline_god_file.py, from the reference tree) and running its pure-PyTorch UltraGauss
fallback (_render_ultragauss_torch_fallback) on the CPU for a small seeded case, with the
gradients of an adjoint-weighted sum of the image. Runs on any machine that has the reference
tree; usage from the repository root:
    python tests/golden/make_dense_fallback_golden.py [--reference /path/to/reference] [--out tests/golden]
"""

from __future__ import annotations

import argparse
import os
import importlib.util
import sys
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=Path, default=os.environ.get("US3D_REFERENCE"),
                    required=not os.environ.get("US3D_REFERENCE"),
                    help="reference checkout (default: $US3D_REFERENCE)")
    ap.add_argument("--out", type=Path, default=Path(__file__).resolve().parent)
    a = ap.parse_args()
    spec = importlib.util.spec_from_file_location("pipeline_god_file", a.reference / "pipeline_god_file.py")
    pgf = importlib.util.module_from_spec(spec)
    sys.modules["pipeline_god_file"] = pgf  # its dataclasses look their module up
    spec.loader.exec_module(pgf)

    g = torch.Generator().manual_seed(0)
    G, H, W = 300, 20, 24
    cfg = pgf.GodConfig(image_height=H, image_width=W, device="cpu")
    init_means = torch.rand((G, 3), generator=g) * 10.0
    init_int = torch.rand((G, 1), generator=g)
    params = pgf.GaussianParameters(cfg, init_means, init_int)
    with torch.no_grad():  # move away from the isotropic initialisation
        params.raw_precision_tril.add_(0.3 * torch.randn((G, 6), generator=g))
        params.raw_opacities.add_(torch.randn((G, 1), generator=g))
    u, v = torch.meshgrid(torch.arange(H, dtype=torch.float32), torch.arange(W, dtype=torch.float32), indexing="ij")
    pixels = torch.stack([v.reshape(-1) * 0.4 + 0.5, u.reshape(-1) * 0.45 + 0.3, torch.full((H * W,), 5.0)], 1)
    out = pgf._render_ultragauss_torch_fallback(params, {"pixel_positions_world": pixels}, cfg)
    adj = torch.randn((1, H, W), generator=g)
    (out.image * adj).sum().backward()
    c = lambda t: t.detach().numpy()  # noqa: E731
    np.savez_compressed(a.out / "dense_fallback_small.npz", means=c(params.means),
                        raw_precision_tril=c(params.raw_precision_tril), raw_opacities=c(params.raw_opacities),
                        raw_intensities=c(params.raw_intensities), pixels=c(pixels), H=H, W=W,
                        diag_beta=np.float64(cfg.ultragauss_diag_beta), adjoint=c(adj), image=c(out.image),
                        alpha=c(out.extras["alpha_image"]), d_means=c(params.means.grad),
                        d_tril=c(params.raw_precision_tril.grad), d_opacities=c(params.raw_opacities.grad),
                        d_intensities=c(params.raw_intensities.grad))
    print("wrote", a.out / "dense_fallback_small.npz")


if __name__ == "__main__":
    main()
