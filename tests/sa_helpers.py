"""Helpers for the slice-adapted 3DGS tests."""

from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def sa_golden_names():
    return sorted(p.stem.split("_", 2)[2] for p in GOLDEN.glob("slice_adapted_*.npz"))


def load_sa(name):
    p = GOLDEN / f"slice_adapted_{name}.npz"
    if not p.exists():
        import pytest

        pytest.skip(f"golden fixture {p.name} not generated")
    return dict(np.load(p))


def run_b200_sa(fx, device):
    import torch

    from us3d_b200 import slice_adapted as SA

    t = lambda k: torch.as_tensor(fx[k]).to(device).contiguous()  # noqa: E731
    H, W, hw, hh, rs = int(fx["H"]), int(fx["W"]), float(fx["half_width"]), float(fx["half_height"]), float(fx["radius_sigma"])
    args = (t("means2d"), t("inv2d"), t("weights"), t("colors"))
    image, alpha, b = SA.bounded_forward(H, W, hw, hh, *args, rs)
    ids, starts, ends = SA.export_bins(b)
    dm, di, dw, dc = SA.bounded_backward(b, hw, hh, *args, t("grad_image"), t("grad_alpha"), rs)
    torch.cuda.synchronize()
    c = lambda x: x.detach().cpu().numpy()  # noqa: E731
    return dict(image=c(image), alpha=c(alpha), sorted_ids=c(ids), range_start=c(starts), range_end=c(ends),
                d_means=c(dm), d_inv=c(di), d_weights=c(dw), d_colors=c(dc))
