"""Shared helpers for the UltraGauss tests."""

from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    den = np.linalg.norm(b)
    num = np.linalg.norm(a - b)
    return float(num / den) if den > 0 else float(num)


def load_golden(name):
    p = GOLDEN / f"ultragauss_{name}.npz"
    if not p.exists():
        import pytest

        pytest.skip(f"golden fixture {p.name} not generated")
    return dict(np.load(p))


def golden_names():
    return sorted(p.stem.split("_", 1)[1] for p in GOLDEN.glob("ultragauss_*.npz"))


def run_b200(fx, device, frames_override=None, capacity=None):
    """Runs bin + forward + backward of the B200 library on one golden-style case."""
    import torch

    from us3d_b200 import ultragauss as UG

    t = lambda k: torch.as_tensor(fx[k]).to(device).contiguous()  # noqa: E731
    geo = fx["geo"]
    spec = UG.SliceSpec(int(fx["H"]), int(fx["W"]), float(geo[12]), float(geo[13]), float(geo[14]), float(geo[15]),
                        torch.as_tensor(geo[0:3]), torch.as_tensor(geo[3:6]), torch.as_tensor(geo[6:9]),
                        torch.as_tensor(geo[9:12]))
    frames = UG.build_frame_table([spec], device)
    means, tril, op, it, pix = t("means"), t("precision_tril"), t("opacities"), t("intensities"), t("pixels")
    b = UG.bin_gaussians(means, tril, op, it, frames, float(fx["chi2"]), float(fx["beta"]), bool(fx["sort_by_depth"]),
                         capacity=capacity)
    image, alpha, depth, counts = UG.forward(b, pix, float(fx["bg_alpha"]), float(fx["bg_intensity"]))
    keys, vals, rs, re = UG.export_bins(b, 0)
    offsets, indices = UG.pixel_csr(b, pix, counts)
    dm, dt, do, di = UG.backward(b, pix, t("d_image"), t("d_alpha"), t("d_depth"), alpha, float(fx["bg_alpha"]),
                                 float(fx["bg_intensity"]))
    torch.cuda.synchronize()
    c = lambda x: x.detach().cpu().numpy()  # noqa: E731
    return dict(keys=c(keys), values=c(vals), range_start=c(rs), range_end=c(re), counts=c(counts),
                offsets=c(offsets), indices=c(indices), image=c(image), alpha=c(alpha), depth=c(depth),
                d_means=c(dm), d_tril=c(dt), d_opacity=c(do), d_intensity=c(di), binning=b)
