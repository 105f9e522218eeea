"""The seeded synthetic scenes: the precision factors written out elementwise agree with the
batched linear-algebra construction, and a scene does not depend on the number of CPU threads
(every number is produced by elementwise operations in a fixed order)."""

from __future__ import annotations

import torch

from us3d_b200 import scenes


def test_precision_tril_matches_cholesky():
    g = torch.Generator().manual_seed(3)
    n, beta = 20000, 1e-4
    s = torch.exp(0.4 * torch.randn((n, 3), generator=g, dtype=torch.float64))
    q = torch.randn((n, 4), generator=g, dtype=torch.float64)
    q = q / q.norm(dim=-1, keepdim=True)
    got = scenes.precision_tril_from_scales_quats(s, q, beta).double()
    R = scenes.quat_to_rot(q)
    lam = R @ torch.diag_embed(1.0 / (s * s)) @ R.transpose(-1, -2)
    L = torch.linalg.cholesky(lam)
    d = torch.diagonal(L, dim1=-2, dim2=-1)
    raw = (d - beta).clamp_min(1e-8).sqrt()
    want = torch.stack([raw[:, 0], L[:, 1, 0], L[:, 2, 0], raw[:, 1], L[:, 2, 1], raw[:, 2]], dim=1)
    assert torch.allclose(got, want, rtol=1e-6, atol=1e-6)


def test_scene_independent_of_thread_count():
    before = torch.get_num_threads()
    try:
        out = []
        for threads in (1, 4):
            torch.set_num_threads(threads)
            sc = scenes.make_scene(50000, seed=5)
            out.append((sc.means, sc.scales, sc.quats, sc.opacities, sc.intensities, sc.precision_tril))
    finally:
        torch.set_num_threads(before)
    for a, b in zip(*out):
        assert torch.equal(a, b)
