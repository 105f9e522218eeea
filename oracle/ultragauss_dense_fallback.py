"""TEST INFRASTRUCTURE ONLY: restatement of the reference's pure-PyTorch UltraGauss fallback
(``_render_ultragauss_torch_fallback``, pipeline_god_file.py:556-603), the path the reference
runs when its CUDA module is absent or on the CPU. It is a dense model without the mapper's
windows, chi-square cut or 1e-8 skip (every pixel against every Gaussian, the exponent clamped
to [-60, 0]), so it is not a parity target for the CUDA renderer; it is timed as the
reference's own CPU baseline at the survey's config-1 size.

Steps, as the reference takes them: L lower-triangular with diagonal raw^2 + beta and the raw
off-diagonals (pipeline_god_file.py:567-575), precision L L^T, sigmoid-activated opacities and
intensities (GaussianParameters, :368-372); per chunk of pixels (2048 on the CPU) and of
Gaussians (512): q = d^T Lambda d, w = exp(clamp(-q/2, -60, 0)) * opacity, numerator
sum w * intensity, denominator sum w; image = clamp01(num / max(den + 1e-6, 1e-8)).
"""

from __future__ import annotations

import torch


def render_dense(means: torch.Tensor, raw_tril: torch.Tensor, raw_opacities: torch.Tensor,
                 raw_intensities: torch.Tensor, pixels: torch.Tensor, diag_beta: float, height: int, width: int,
                 pixel_chunk: int = 2048, gauss_chunk: int = 512):
    """(image (1,H,W), alpha (1,H,W)); differentiable with torch autograd."""
    G = means.shape[0]
    L = torch.zeros((G, 3, 3), dtype=raw_tril.dtype, device=raw_tril.device)
    L[:, 0, 0] = raw_tril[:, 0].square() + diag_beta
    L[:, 1, 0] = raw_tril[:, 1]
    L[:, 2, 0] = raw_tril[:, 2]
    L[:, 1, 1] = raw_tril[:, 3].square() + diag_beta
    L[:, 2, 1] = raw_tril[:, 4]
    L[:, 2, 2] = raw_tril[:, 5].square() + diag_beta
    lam = L @ L.transpose(-1, -2)
    opac = torch.sigmoid(raw_opacities).reshape(-1)
    inten = torch.sigmoid(raw_intensities).reshape(-1)
    images, alphas = [], []
    for p0 in range(0, pixels.shape[0], pixel_chunk):
        p = pixels[p0:p0 + pixel_chunk]
        num = torch.zeros((p.shape[0],), dtype=pixels.dtype)
        den = torch.zeros_like(num)
        for g0 in range(0, G, gauss_chunk):
            g1 = min(g0 + gauss_chunk, G)
            d = p[:, None, :] - means[None, g0:g1, :]
            q = torch.einsum("pgi,gij,pgj->pg", d, lam[g0:g1], d)
            w = torch.exp(torch.clamp(-0.5 * q, min=-60.0, max=0.0)) * opac[g0:g1].view(1, -1)
            num = num + (w * inten[g0:g1].view(1, -1)).sum(dim=1)
            den = den + w.sum(dim=1)
        images.append(num / torch.clamp(den + 1.0e-6, min=1.0e-8))
        alphas.append(den)
    image = torch.cat(images).view(height, width).unsqueeze(0).clamp(0.0, 1.0)
    return image, torch.cat(alphas).view(1, height, width)
