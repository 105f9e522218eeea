"""The restatement of the reference's dense PyTorch UltraGauss fallback (the reference's own
CPU path, timed by bench.py as its CPU baseline at config-1 size) against golden vectors made
by running the reference's pipeline_god_file._render_ultragauss_torch_fallback itself
(tests/golden/make_dense_fallback_golden.py): image, alpha and the gradients of an
adjoint-weighted image sum."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import torch

GOLDEN = Path(__file__).resolve().parent / "golden" / "dense_fallback_small.npz"


def test_dense_fallback_matches_reference_vectors():
    from oracle.ultragauss_dense_fallback import render_dense

    fx = np.load(GOLDEN)
    t = {k: torch.from_numpy(fx[k]).requires_grad_(True) for k in
         ("means", "raw_precision_tril", "raw_opacities", "raw_intensities")}
    img, alpha = render_dense(t["means"], t["raw_precision_tril"], t["raw_opacities"], t["raw_intensities"],
                              torch.from_numpy(fx["pixels"]), float(fx["diag_beta"]), int(fx["H"]), int(fx["W"]))
    (img * torch.from_numpy(fx["adjoint"])).sum().backward()
    np.testing.assert_allclose(img.detach().numpy(), fx["image"], rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(alpha.detach().numpy(), fx["alpha"], rtol=1e-6, atol=1e-7)
    for k, g in (("means", "d_means"), ("raw_precision_tril", "d_tril"), ("raw_opacities", "d_opacities"),
                 ("raw_intensities", "d_intensities")):
        np.testing.assert_allclose(t[k].grad.numpy(), fx[g], rtol=1e-5, atol=1e-7 * np.abs(fx[g]).max())
