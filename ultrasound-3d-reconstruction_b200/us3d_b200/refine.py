"""Densification and pruning of UltraGauss Gaussians during training.

The reference trains a fixed set of Gaussians (pipeline_god_file.py:737-764 never adds or
removes any); the refinement below is the one the UltraG-Ray paper describes
(ops/ultragray_renderer/old ultragray reproduct guide.md:161-167: every 2500 iterations from
1k to 20k, importance from accumulated gradients, small Gaussians duplicated and large ones
split, pruning of scales below 5e-5 or above 5 mm, at most 500k Gaussians), applied to the
UltraGauss parameterisation. It has no counterpart in the reference's code, hence no parity
target; its rules are stated and tested here.

Statistics are accumulated on the device every step (``us3d_ug_refine_stats``: |dL/dmean| and
the number of steps in which a Gaussian received a gradient). A refinement step, on the
device with PyTorch tensor operations (it runs once every few thousand steps):

* scale: the principal standard deviations of Sigma = (L L^T)^-1, L the lower-triangular factor
  with diagonal raw^2 + beta (the renderer's precision parameterisation);
* prune: non-finite parameters, largest scale > ``prune_max_scale_mm``, smallest scale < ``prune_min_scale_mm`` or
  opacity sigmoid(raw) < ``min_opacity``;
* densify (not pruned, mean importance per visited step > ``grad_threshold``, or among the top
  ``densify_fraction`` of the visited Gaussians when that is set): largest scale
  <= ``split_scale_mm`` -> clone (an exact copy is added); larger -> split (replaced by two
  children with means drawn from N(mean, Sigma) and Sigma shrunk by ``split_factor``^2, i.e.
  L scaled by ``split_factor``, other attributes copied);
* the number of Gaussians is capped at ``max_gaussians`` (densification candidates taken in
  decreasing importance);
* kept Gaussians keep their Adam moments; new ones start from zero moments.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional

import torch

from . import _lib
from .ultragauss import _ptr, _stream


@dataclass
class RefineConfig:
    every: int = 2500
    start: int = 1000
    stop: int = 20000
    grad_threshold: float = 2.0e-4
    split_scale_mm: float = 1.0
    split_factor: float = 1.6
    prune_min_scale_mm: float = 5.0e-5
    prune_max_scale_mm: float = 5.0
    min_opacity: float = 0.005
    max_gaussians: int = 500000
    diag_beta: float = 1.0e-4
    # When set, the importance threshold of each refinement is the (1 - fraction) quantile of
    # the scores of the visited, unpruned Gaussians (the top ``densify_fraction`` are densified)
    # instead of ``grad_threshold``: |dL/dmean| scales with how the loss is normalised (pixels
    # and frames per step), a quantile does not.
    densify_fraction: Optional[float] = None

    def due(self, step: int) -> bool:
        """Whether a refinement follows training step ``step`` (counted from 1)."""
        return self.start <= step <= self.stop and step % self.every == 0


class RefineStats:
    """Per-Gaussian importance (sum of |dL/dmean|) and visit counts on the device."""

    def __init__(self, n: int, device):
        self.importance = torch.zeros(n, dtype=torch.float32, device=device)
        self.visits = torch.zeros(n, dtype=torch.int32, device=device)

    def accumulate(self, grad_means: torch.Tensor) -> None:
        n = self.importance.numel()
        if grad_means.shape != (n, 3) or not grad_means.is_contiguous():
            raise ValueError(f"grad_means must be a contiguous ({n}, 3) tensor")
        _lib.check(_lib.call("us3d_ug_refine_stats", _ptr(grad_means), n, _ptr(self.importance), _ptr(self.visits),
                             _stream()), "us3d_ug_refine_stats")

    def score(self) -> torch.Tensor:
        return self.importance / self.visits.clamp_min(1).float()


def factor_from_raw(raw_tril: torch.Tensor, beta: float) -> torch.Tensor:
    """Lower-triangular L (G,3,3) of the precision L L^T from the raw (G,6) parameters."""
    G = raw_tril.shape[0]
    L = torch.zeros((G, 3, 3), dtype=raw_tril.dtype, device=raw_tril.device)
    L[:, 0, 0] = raw_tril[:, 0].square() + beta
    L[:, 1, 0] = raw_tril[:, 1]
    L[:, 2, 0] = raw_tril[:, 2]
    L[:, 1, 1] = raw_tril[:, 3].square() + beta
    L[:, 2, 1] = raw_tril[:, 4]
    L[:, 2, 2] = raw_tril[:, 5].square() + beta
    return L


def _sym3_largest(M: torch.Tensor) -> torch.Tensor:
    """Largest eigenvalue of symmetric 3x3 matrices (..., 3, 3), closed form: the
    trigonometric solution of the characteristic cubic (q = tr/3, p = sqrt(|M - qI|_F^2 / 6),
    r = det((M - qI) / p) / 2, largest root q + 2p cos(acos(r)/3)); elementwise tensor
    arithmetic, any number of matrices in one pass. The largest root carries no cancellation,
    so its relative error is a few ulps."""
    a, b, c = M[..., 0, 0], M[..., 1, 1], M[..., 2, 2]
    d, e, f = M[..., 0, 1], M[..., 1, 2], M[..., 0, 2]
    q = (a + b + c) / 3.0
    aq, bq, cq = a - q, b - q, c - q
    p = torch.sqrt((aq * aq + bq * bq + cq * cq + 2.0 * (d * d + e * e + f * f)) / 6.0)
    safe = torch.where(p > 0, p, torch.ones_like(p))
    ba, bb, bc, bd, be, bf = aq / safe, bq / safe, cq / safe, d / safe, e / safe, f / safe
    det = ba * (bb * bc - be * be) - bd * (bd * bc - be * bf) + bf * (bd * be - bb * bf)
    return q + 2.0 * p * torch.cos(torch.acos((det * 0.5).clamp(-1.0, 1.0)) / 3.0)


def principal_scales(raw_tril: torch.Tensor, beta: float) -> torch.Tensor:
    """(G,3) standard deviations along the principal axes, ascending (NaN where the
    parameters are not finite). With the precision L L^T (L lower triangular, diagonal
    raw^2 + beta): s_min = 1 / sqrt(largest eigenvalue of L L^T), s_max = sqrt(largest
    eigenvalue of the covariance L^-T L^-1) and s_mid from s_min s_mid s_max = 1 / det L. Only
    largest eigenvalues are taken, in closed form (no batched solver: the library one refuses
    millions of matrices in one call), so each scale keeps its relative accuracy however
    elongated the Gaussian is."""
    L = factor_from_raw(raw_tril.double(), beta)
    l00, l10, l11, l20, l21, l22 = L[:, 0, 0], L[:, 1, 0], L[:, 1, 1], L[:, 2, 0], L[:, 2, 1], L[:, 2, 2]
    Li = torch.zeros_like(L)  # L^-1, lower triangular
    Li[:, 0, 0] = 1.0 / l00
    Li[:, 1, 1] = 1.0 / l11
    Li[:, 2, 2] = 1.0 / l22
    Li[:, 1, 0] = -l10 / (l00 * l11)
    Li[:, 2, 1] = -l21 / (l11 * l22)
    Li[:, 2, 0] = (l10 * l21 - l11 * l20) / (l00 * l11 * l22)
    s_min = 1.0 / torch.sqrt(_sym3_largest(L @ L.transpose(-1, -2)))
    s_max = torch.sqrt(_sym3_largest(Li.transpose(-1, -2) @ Li))
    s_mid = 1.0 / ((l00 * l11 * l22).abs() * s_min * s_max)
    return torch.stack([s_min, s_mid, s_max], 1).float()


def _raw_from_factor(L: torch.Tensor, beta: float) -> torch.Tensor:
    diag = torch.stack([L[:, 0, 0], L[:, 1, 1], L[:, 2, 2]], 1)
    raw_d = (diag - beta).clamp_min(1e-12).sqrt()
    return torch.stack([raw_d[:, 0], L[:, 1, 0], L[:, 2, 0], raw_d[:, 1], L[:, 2, 1], raw_d[:, 2]], 1)


@torch.no_grad()
def refine(params, optimizer, stats: RefineStats, cfg: RefineConfig,
           generator: Optional[torch.Generator] = None) -> dict:
    """One refinement of ``params`` (train.UltraGaussParameters) in place, with the Adam
    moments of ``optimizer`` (train.Adam over params.tensors()) carried along and ``stats``
    reset. Returns the counts {kept, pruned, cloned, split, total}."""
    means, tril = params.means, params.raw_precision_tril
    raw_o, raw_i = params.raw_opacities, params.raw_intensities
    G = means.shape[0]
    dev = means.device
    scales = principal_scales(tril, cfg.diag_beta)
    s_min, s_max = scales[:, 0], scales[:, 2]
    opac = torch.sigmoid(raw_o.reshape(-1))
    prune = (s_max > cfg.prune_max_scale_mm) | (s_min < cfg.prune_min_scale_mm) | (opac < cfg.min_opacity)
    prune |= ~(torch.isfinite(scales).all(1) & torch.isfinite(means).all(1) & torch.isfinite(opac))
    score = stats.score()
    threshold = cfg.grad_threshold
    if cfg.densify_fraction is not None:
        sv = torch.sort(score[(~prune) & (stats.visits > 0)]).values
        n, m = sv.numel(), int(math.ceil(sv.numel() * float(cfg.densify_fraction)))
        # the m highest scores lie strictly above sv[n - m - 1] (ties with it are left out)
        threshold = float("inf") if m <= 0 else (float("-inf") if m >= n else float(sv[n - m - 1]))
    cand = (~prune) & (score > threshold)
    budget = max(0, int(cfg.max_gaussians) - int((~prune).sum()))
    idx = cand.nonzero().flatten()
    if idx.numel() > budget:  # each candidate adds one Gaussian (a clone, or two children for one)
        keep_top = torch.argsort(score[idx], descending=True, stable=True)[:budget]
        idx = idx[keep_top.sort().values]
    dens = torch.zeros(G, dtype=torch.bool, device=dev)
    dens[idx] = True
    clone = dens & (s_max <= cfg.split_scale_mm)
    split = dens & (s_max > cfg.split_scale_mm)
    keep = (~prune) & (~split)

    # children of the split Gaussians: means ~ N(mean, Sigma), x = L^-T z has covariance Sigma
    sp = split.nonzero().flatten()
    L = factor_from_raw(tril[sp].double(), cfg.diag_beta)
    z = torch.randn((2, sp.numel(), 3, 1), generator=generator, device=dev, dtype=torch.float64)
    offs = torch.linalg.solve_triangular(L.transpose(-1, -2).unsqueeze(0).expand(2, -1, -1, -1), z,
                                         upper=True).squeeze(-1)
    child_means = (means[sp].double().unsqueeze(0) + offs).reshape(-1, 3).float()
    child_tril = _raw_from_factor(L * cfg.split_factor, cfg.diag_beta).float().repeat(2, 1)
    cl = clone.nonzero().flatten()
    new_means = torch.cat([means[keep], means[cl], child_means])
    new_tril = torch.cat([tril[keep], tril[cl], child_tril])
    new_o = torch.cat([raw_o[keep], raw_o[cl], raw_o[sp].repeat(2, 1)])
    new_i = torch.cat([raw_i[keep], raw_i[cl], raw_i[sp].repeat(2, 1)])
    n_new = int(cl.numel() + 2 * sp.numel())

    def moments(t_list):
        out = []
        for t in t_list:
            kept = t[keep]
            out.append(torch.cat([kept, torch.zeros((n_new,) + tuple(t.shape[1:]), dtype=t.dtype, device=dev)])
                       .contiguous())
        return out

    optimizer.exp_avg = moments(optimizer.exp_avg)
    optimizer.exp_avg_sq = moments(optimizer.exp_avg_sq)
    params.means = new_means.contiguous()
    params.raw_precision_tril = new_tril.contiguous()
    params.raw_opacities = new_o.contiguous()
    params.raw_intensities = new_i.contiguous()
    optimizer.params = params.tensors()
    n = params.means.shape[0]
    stats.importance = torch.zeros(n, dtype=torch.float32, device=dev)
    stats.visits = torch.zeros(n, dtype=torch.int32, device=dev)
    return {"kept": int(keep.sum()), "pruned": int(prune.sum()), "cloned": int(cl.numel()), "split": int(sp.numel()),
            "total": n}
