"""Generates tests/golden/ultragauss_*.npz from the reference's own UltraGauss CUDA build.

Needs a CUDA GPU and the reference build in oracle/_ref (python oracle/build_ref.py).
Inputs are the seeded synthetic scenes of us3d_b200.scenes; outputs are exactly what the
reference's MapperForwardCUDA / ShaderForwardCUDA / ShaderBackwardCUDA return, plus its
private sorted keys and tile ranges (oracle/ref_harness/ultragauss_keys.cu).

Usage (on a GPU machine, from the repository root):
    python tests/golden/make_ultragauss_golden.py [--out tests/golden]
"""

from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]
sys.path[:0] = [str(ROOT), str(ROOT / "ultrasound-3d-reconstruction_b200"), str(ROOT / "oracle" / "_ref")]

import ultragauss_ref_C as REF  # noqa: E402
import ultragauss_ref_keys as REFK  # noqa: E402

from us3d_b200 import scenes  # noqa: E402


def pad4(t):
    return torch.nn.functional.pad(t, (0, 1)).contiguous()


def case_inputs(name):
    if name == "c1":
        sc = scenes.make_scene(4096, seed=0)
        fr = scenes.linear_sweep(16, 128, 128, 0.3, seed=0)[8]
        p = dict(H=128, W=128, dlat=0.3, dax=0.3, near=0.0, coloff=fr.lateral_col_offset, chi2=7.815, beta=1e-4,
                 sort=True, bg_a=1e-6, bg_i=0.0)
        return sc, fr.origin, fr.axis_lat, fr.axis_ax, fr.axis_ele, fr.pixels, p
    if name == "ragged":
        sc = scenes.make_scene(1500, seed=1, cube_mm=40.0, log_scale_mean=0.3)
        H, W, dlat, dax, near, coloff = 50, 70, 0.6, 0.4, 3.0, 10.5
        origin = torch.tensor([8.0, 1.0, 20.5])
        lat = torch.tensor([1.0, 0.0, 0.0])
        c, s = np.cos(0.2), np.sin(0.2)
        ax = torch.tensor([0.0, float(c), float(s)])
        ele = torch.tensor([0.0, float(-s), float(c)])
        pix = scenes.slice_pixels(origin, lat, ax, H, W, dlat, dax, near, coloff)
        p = dict(H=H, W=W, dlat=dlat, dax=dax, near=near, coloff=coloff, chi2=9.0, beta=1e-4, sort=False, bg_a=0.05,
                 bg_i=0.3)
        return sc, origin, lat, ax, ele, pix, p
    if name == "tiny":
        means = torch.tensor([[5.0, 5.0, 0.2], [30.0, 8.0, 0.0], [12.0, 20.0, 9.0], [-40.0, 5.0, 0.0],
                              [7.0, 7.0, -0.5]])
        scales = torch.tensor([[2.0, 1.0, 1.0], [3.0, 3.0, 0.5], [1.0, 1.0, 1.0], [1.0, 1.0, 1.0], [0.2, 4.0, 1.5]])
        quats = torch.nn.functional.normalize(torch.tensor([[1.0, 0, 0, 0], [0.9, 0.1, 0.2, 0.3], [1.0, 0, 0, 0],
                                                            [1.0, 0, 0, 0], [0.5, 0.5, 0.5, 0.5]]), dim=-1)
        sc = scenes.GaussianScene(means, scales, quats, torch.tensor([0.9, 0.5, 0.7, 0.8, 0.3]),
                                  torch.tensor([0.2, 0.9, 0.5, 0.4, 1.0]),
                                  scenes.precision_tril_from_scales_quats(scales, quats))
        H, W = 24, 40
        origin = torch.tensor([0.0, 0.0, 0.0])
        lat, ax, ele = torch.eye(3)
        pix = scenes.slice_pixels(origin, lat, ax, H, W, 1.0, 1.0, 0.0, 0.0)
        p = dict(H=H, W=W, dlat=1.0, dax=1.0, near=0.0, coloff=0.0, chi2=7.815, beta=1e-4, sort=True, bg_a=0.0,
                 bg_i=0.0)
        return sc, origin, lat, ax, ele, pix, p
    raise KeyError(name)


def run_case(name):
    sc, origin, lat, ax, ele, pix, p = case_inputs(name)
    dev = torch.device("cuda")
    means = sc.means.to(dev)
    tril = sc.precision_tril.to(dev).contiguous()
    op = sc.opacities.to(dev)
    it = sc.intensities.to(dev)
    o, l, a, e = (x.to(dev).float().contiguous() for x in (origin, lat, ax, ele))
    pixd = pix.to(dev)
    mp, pp = pad4(means), pad4(pixd)
    counts, offsets, indices = REF.MapperForwardCUDA(pp, mp, tril, o, l, a, e, p["H"], p["W"], p["dlat"], p["dax"],
                                                     p["near"], p["coloff"], p["chi2"], p["sort"], p["beta"])
    attr = torch.stack([op, it], dim=1).contiguous()
    image, alpha, depth, sic = REF.ShaderForwardCUDA(attr, mp, tril, pp, o, e, offsets, counts, indices, p["bg_a"],
                                                     p["bg_i"], p["chi2"], p["beta"])
    g = torch.Generator().manual_seed(123)
    P = pix.shape[0]
    dI = torch.randn(P, generator=g)
    dA = 0.3 * torch.randn(P, generator=g)
    dD = 0.05 * torch.randn(P, generator=g)
    dm, dt, da = REF.ShaderBackwardCUDA(dI.to(dev), dA.to(dev), dD.to(dev), attr, mp, tril, pp, o, e, offsets, counts,
                                        indices, sic, alpha, p["bg_a"], p["bg_i"], p["chi2"], p["beta"])
    touched, rects, depths, keys, vals, rs, re = REFK.RefBinning(mp, tril, o, l, a, e, p["H"], p["W"], p["dlat"],
                                                                 p["dax"], p["near"], p["coloff"], p["chi2"],
                                                                 p["sort"], p["beta"])
    torch.cuda.synchronize()
    c = lambda t: t.detach().cpu().numpy()  # noqa: E731
    geo = np.concatenate([c(o), c(l), c(a), c(e), np.array([p["dlat"], p["dax"], p["near"], p["coloff"]], np.float32)])
    return dict(
        means=c(means), precision_tril=c(tril), opacities=c(op), intensities=c(it), pixels=c(pixd),
        geo=geo.astype(np.float32), H=p["H"], W=p["W"], chi2=np.float32(p["chi2"]), beta=np.float32(p["beta"]),
        sort_by_depth=int(p["sort"]), bg_alpha=np.float32(p["bg_a"]), bg_intensity=np.float32(p["bg_i"]),
        d_image=c(dI), d_alpha=c(dA), d_depth=c(dD),
        ref_touched=c(touched), ref_rects=c(rects), ref_depths=c(depths), ref_keys=c(keys), ref_values=c(vals),
        ref_range_start=c(rs), ref_range_end=c(re), ref_counts=c(counts), ref_offsets=c(offsets),
        ref_indices=c(indices), ref_image=c(image), ref_alpha=c(alpha), ref_depth=c(depth),
        ref_d_means=c(dm)[:, :3], ref_d_tril=c(dt), ref_d_opacity=c(da)[:, 0], ref_d_intensity=c(da)[:, 1],
    )


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", type=Path, default=Path(__file__).resolve().parent)
    a = ap.parse_args()
    a.out.mkdir(parents=True, exist_ok=True)
    for name in ("c1", "ragged", "tiny"):
        d = run_case(name)
        np.savez_compressed(a.out / f"ultragauss_{name}.npz", **d)
        print(name, {k: getattr(v, "shape", v) for k, v in d.items() if k.startswith("ref_")})


if __name__ == "__main__":
    main()
