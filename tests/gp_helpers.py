"""Helpers for the GaussianPile tests."""

from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def gp_golden_names():
    return sorted(p.stem.split("_", 1)[1] for p in GOLDEN.glob("gaussianpile_*.npz"))


def load_gp(name):
    p = GOLDEN / f"gaussianpile_{name}.npz"
    if not p.exists():
        import pytest

        pytest.skip(f"golden fixture {p.name} not generated")
    return dict(np.load(p))


def run_b200_gp(fx, device):
    import torch

    from us3d_b200 import gaussianpile as GP

    t = lambda k: torch.as_tensor(fx[k]).to(device).float().contiguous()  # noqa: E731
    m = fx["meta"].tolist()
    img, b = GP.forward(t("means"), t("scales"), t("quats"), t("opacities").reshape(-1), t("intensities").reshape(-1),
                        t("pose").reshape(16), t("grid"), t("params"), int(fx["H"]), int(fx["W"]), m[2], m[3], m[4],
                        int(m[5]), m[8], bool(m[9]))
    ids, rs, re, rects = GP.export_bins(b)
    grads = GP.backward(b, t("grad_image"), bool(fx["pose_grad"]))
    torch.cuda.synchronize()
    c = lambda x: x.detach().cpu().numpy()  # noqa: E731
    out = dict(image=c(img), sorted_ids=c(ids), range_start=c(rs), range_end=c(re), rects=c(rects))
    for k, v in zip(("d_means", "d_scales", "d_quats", "d_opacity", "d_intensity", "d_pose"), grads):
        out[k] = c(v)
    return out
