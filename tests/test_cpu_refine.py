"""Refinement rules (densify / prune) of us3d_b200.refine on the CPU, on planted Gaussians:
pruning by scale and opacity, cloning of important small Gaussians, splitting of important
large ones (children drawn around the parent with the precision factor scaled by the split
factor), the cap on the number of Gaussians, and the Adam moments carried along."""

from __future__ import annotations

import math

import torch


def _iso_raw(scale_mm, beta=1e-4):
    d = math.sqrt(max(1.0 / scale_mm - beta, 1e-12))
    return [d, 0.0, 0.0, d, 0.0, d]


def _setup(max_gaussians=100):
    from us3d_b200.refine import RefineConfig, RefineStats
    from us3d_b200.train import UltraGaussParameters

    scales = [0.5, 0.5, 2.0, 2.0, 10.0, 1e-6, 0.5, 0.5]
    opac = [0.5, 0.5, 0.5, 0.5, 0.5, 0.5, 0.001, 0.5]
    imp = [1.0, 0.0, 1.0, 0.0, 1.0, 1.0, 1.0, 2.0]
    G = len(scales)
    means = torch.arange(G * 3, dtype=torch.float32).reshape(G, 3)
    tril = torch.tensor([_iso_raw(s) for s in scales], dtype=torch.float32)
    logit = lambda p: math.log(p / (1 - p))  # noqa: E731
    params = UltraGaussParameters(means, tril, torch.tensor([[logit(p)] for p in opac]),
                                  torch.linspace(-1, 1, G).reshape(G, 1))
    stats = RefineStats.__new__(RefineStats)
    stats.importance = torch.tensor(imp)
    stats.visits = torch.ones(G, dtype=torch.int32)

    class Opt:  # the moments of train.Adam, without a GPU
        pass

    opt = Opt()
    opt.exp_avg = [torch.full_like(t, 7.0) for t in params.tensors()]
    opt.exp_avg_sq = [torch.full_like(t, 3.0) for t in params.tensors()]
    cfg = RefineConfig(grad_threshold=0.5, split_scale_mm=1.0, max_gaussians=max_gaussians)
    return params, opt, stats, cfg, means, tril


def test_refine_rules():
    from us3d_b200.refine import factor_from_raw, refine

    params, opt, stats, cfg, means, tril = _setup()
    out = refine(params, opt, stats, cfg, torch.Generator().manual_seed(0))
    # pruned: 4 (scale 10 > 5), 5 (scale 1e-6 < 5e-5), 6 (opacity 0.001); split: 2; cloned: 0, 7
    assert out == {"kept": 4, "pruned": 3, "cloned": 2, "split": 1, "total": 8}
    kept, clones = [0, 1, 3, 7], [0, 7]
    assert torch.equal(params.means[:4], means[kept])
    assert torch.equal(params.means[4:6], means[clones])
    assert torch.equal(params.raw_precision_tril[:6], tril[kept + clones])
    L_parent = factor_from_raw(tril[2:3].double(), cfg.diag_beta)
    L_child = factor_from_raw(params.raw_precision_tril[6:].double(), cfg.diag_beta)
    assert torch.allclose(L_child, (cfg.split_factor * L_parent).expand(2, 3, 3), rtol=1e-5, atol=1e-6)
    assert ((params.means[6:] - means[2]).norm(dim=1) < 10.0).all()  # within 5 sigma of the parent
    for m in opt.exp_avg:
        assert (m[:4] == 7.0).all() and (m[4:] == 0.0).all()
    assert stats.importance.shape == (8,) and int(stats.visits.sum()) == 0


def test_refine_cap_keeps_most_important():
    from us3d_b200.refine import refine

    params, opt, stats, cfg, means, tril = _setup(max_gaussians=6)
    out = refine(params, opt, stats, cfg, torch.Generator().manual_seed(0))
    # 5 survive pruning, room for one more: the most important candidate (7, a clone)
    assert out == {"kept": 5, "pruned": 3, "cloned": 1, "split": 0, "total": 6}
    assert torch.equal(params.means[5], means[7])


def test_refine_schedule():
    from us3d_b200.refine import RefineConfig

    c = RefineConfig(every=2500, start=1000, stop=20000)
    assert [s for s in range(1, 25001) if c.due(s)] == list(range(2500, 20001, 2500))


def test_principal_scales_closed_form_and_non_finite():
    """Scales in closed form (no batched solver: the library one refuses millions of matrices
    in one call): against LAPACK on random factors including Gaussians elongated 10^5 : 1,
    each scale to 1e-9 relative; a Gaussian with a non-finite factor gets NaN scales (and is
    pruned by refine) without disturbing the others."""
    from us3d_b200 import refine as R

    g = torch.Generator().manual_seed(3)
    tril = torch.randn((5000, 6), generator=g, dtype=torch.float64) * torch.tensor([3.0, 1, 1, 0.2, 1, 0.05])
    L = R.factor_from_raw(tril, 1e-4)
    ref = (1.0 / torch.linalg.eigvalsh(L @ L.transpose(-1, -2)).sqrt()).flip(-1)
    well = torch.nan_to_num(ref[:, 2] / ref[:, 0], nan=1e30) < 1e4  # LAPACK loses the small eigenvalue beyond
    scales = R.principal_scales(tril.float(), 1e-4)
    assert torch.allclose(scales.double()[well], ref[well], rtol=1e-6)
    s64 = R.principal_scales(tril, 1e-4).double()
    L = R.factor_from_raw(tril, 1e-4)
    # elongated ones against the exact relation s_min s_mid s_max = 1 / det L and the
    # singular values of L^-1 (the covariance's square roots) from an SVD
    sv = torch.linalg.svdvals(torch.linalg.inv(L)).flip(-1)
    assert torch.allclose(s64[:, 2], sv[:, 2], rtol=1e-6)
    assert torch.allclose(s64[:, 0], sv[:, 0], rtol=1e-6)
    assert (scales[:, 0] <= scales[:, 1]).all() and (scales[:, 1] <= scales[:, 2]).all()
    assert (s64[:, 2] / s64[:, 0]).max() > 1e5
    bad = tril.float().clone()
    bad[5, 2] = float("nan")
    s = R.principal_scales(bad, 1e-4)
    assert torch.isnan(s[5]).all()
    keep = torch.arange(5000) != 5
    assert torch.equal(s[keep], scales[keep])


def test_refine_densify_fraction():
    """With densify_fraction the threshold is a quantile of the visited, unpruned Gaussians'
    scores: of the five survivors (scores 1, 0, 1, 0, 2) the top 20 % is Gaussian 7 alone, the
    top 60 % adds the two with score 1 (0 clone, 2 split)."""
    from us3d_b200.refine import refine

    params, opt, stats, cfg, means, tril = _setup()
    cfg.grad_threshold = 1e9  # ignored when a fraction is given
    cfg.densify_fraction = 0.2
    out = refine(params, opt, stats, cfg, torch.Generator().manual_seed(0))
    assert out == {"kept": 5, "pruned": 3, "cloned": 1, "split": 0, "total": 6}
    params, opt, stats, cfg, means, tril = _setup()
    cfg.densify_fraction = 0.6
    out = refine(params, opt, stats, cfg, torch.Generator().manual_seed(0))
    assert out == {"kept": 4, "pruned": 3, "cloned": 2, "split": 1, "total": 8}
