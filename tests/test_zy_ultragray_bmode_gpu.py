"""UltraGray at the B-mode workload's scale and its finite-difference gradient check.

Workload: 1,000,000 Gaussians in a 40 x 60 x 64 mm box (us3d_b200.scenes.make_bmode_scene:
reflectivity U(0,1) with 5 % strong reflectors U(5,10), attenuation logits for 0.5 dB/cm/MHz
at 5 MHz), frames of 512 scanlines x 1024 samples over 60 mm depth from a 40 mm linear array
(scenes.bmode_sweep, 64 frames along the sweep). One frame is checked against the
reference's own CUDA build: ray CSR bit-exact, image <= 1e-5 and gradients <= 1e-4 relative
L2; both are timed (printed). At this size the transmittance checkpoints carry the
transmission product (the per-sample path is compared on a second frame with decreasing
sample depths, which it keeps).

Gradient check: the GPU adjoint against central differences (step 1e-4) of the FP64 oracle
on a 1,024-Gaussian, 64-scanline x 128-sample sub-problem of the same scene, with the
quadrature window radius 0 (the reference's backward differentiates the Gauss-Legendre sum
with the window limits held fixed, which is the exact derivative only without a window).
"""

from __future__ import annotations

import math
import sys
import time
from pathlib import Path

import numpy as np
import pytest
import torch

from ug_helpers import rel_l2

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def _scene_dict(sc, fr, W, H, grad_seed, wr=2.0, rays=None, samples=None, gauss=None):
    """The renderer inputs (ugr_helpers layout) of frame fr, optionally a sub-problem."""
    rays = slice(None) if rays is None else rays
    samples = slice(None) if samples is None else samples
    gauss = slice(None) if gauss is None else gauss
    rng = np.random.default_rng(grad_seed)
    ro = fr.ray_origins[rays].numpy()
    pix = fr.pixels[rays][:, samples].numpy()
    Wd, Hd = pix.shape[0], pix.shape[1]
    u = rng.uniform(0, 1, Wd)
    pert = (np.arcsin(2 * u - 1) / (math.pi / 2) * 0.5).astype(np.float32)
    gimg = rng.normal(size=(Hd, Wd)).astype(np.float32)
    fl = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
    col_off = (W - 1) * 0.5
    if rays != slice(None):
        col_off -= rays.start
    return dict(means=fl(sc.means[gauss].numpy()), scales=fl(sc.scales[gauss].numpy()),
                quats=fl(sc.quats[gauss].numpy()), attenuations=fl(sc.attenuations[gauss].numpy()),
                sh=fl(sc.sh[gauss].numpy()), pixels=fl(pix), ray_o=fl(ro), ray_d=fl(fr.ray_dirs[rays].numpy()),
                origin=fl(fr.origin.numpy()), lat=fl(fr.axis_lat.numpy()), ele=fl(fr.axis_ele.numpy()),
                ax=fl(fr.axis_ax.numpy()), pert=pert, grad_image=gimg, width_mm=float(fr.width_mm * Wd / W),
                near_mm=0.0, col_off=float(col_off), elev_cut=0.0, k_sigma=3.0, wr=float(wr), local=False,
                maxwin=17.0)


def _ref_module():
    p = ROOT / "oracle" / "_ref"
    if not any(p.glob("ultragray_ref_C*.so")):
        pytest.skip("reference build not present")
    sys.path.insert(0, str(p))
    import ultragray_ref_C

    return ultragray_ref_C


def test_ultragray_bmode_scale_against_reference(cuda_device):
    REF = _ref_module()
    import test_ultragray_gpu as T
    from ugr_helpers import run_b200_ugr, run_reference_ugr

    from us3d_b200 import scenes

    from ugr_helpers import SCENE_ARRAYS, params
    from us3d_b200 import ultragray as U

    sc = scenes.make_bmode_scene(1_000_000, seed=0)
    fr = scenes.bmode_sweep(64)[32]
    scene = _scene_dict(sc, fr, 512, 1024, 5)
    out = run_b200_ugr(scene, cuda_device)  # warm-up and result
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    run_b200_ugr(scene, cuda_device)
    t_ours = time.perf_counter() - t0
    # device time of the forward (binning included) and of the backward
    t = {k: torch.as_tensor(scene[k]).to(cuda_device).contiguous() for k in SCENE_ARRAYS}
    p = params(scene)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record()
    _, b = U.forward(t["means"], t["scales"], t["quats"], t["attenuations"], t["sh"], t["pixels"], t["ray_o"],
                     t["ray_d"], t["origin"], t["lat"], t["ele"], t["ax"], t["pert"], p, capacity=out["total"] + 1024)
    ev[1].record()
    U.backward(b, t["quats"], t["pixels"], t["ray_o"], t["ray_d"], t["ele"], t["pert"], t["grad_image"], p)
    ev[2].record()
    ev[2].synchronize()
    print(f"ultragray B-mode device time: forward {ev[0].elapsed_time(ev[1]):.2f} ms, "
          f"backward {ev[1].elapsed_time(ev[2]):.2f} ms")
    t0 = time.perf_counter()
    ref = run_reference_ugr(REF, scene, cuda_device)
    t_ref = time.perf_counter() - t0
    errs = {k: rel_l2(out[k], ref["ref_" + k]) for k in ("image", "d_means", "d_scales", "d_quats", "d_attens", "d_sh")}
    print(f"ultragray B-mode frame (1M Gaussians, 512 x 1024): {out['total']} instances, "
          f"max per ray {int(out['counts'].max())}; fwd+bwd ours {t_ours * 1e3:.1f} ms, reference {t_ref * 1e3:.1f} ms; "
          f"rel-L2 vs reference {errs}")
    T._check(out, ref)


def test_ultragray_nonmonotone_rays_keep_per_sample_path(cuda_device):
    """A scanline whose sample depths decrease somewhere cannot use the checkpoints: the
    frame mixes such rays (samples reversed) with ordinary ones and every ray must still match
    the reference."""
    REF = _ref_module()
    import test_ultragray_gpu as T
    from ugr_helpers import make_scene, run_b200_ugr, run_reference_ugr

    scene = make_scene(20000, 96, 160, 21)
    pix = scene["pixels"].copy()
    pix[::3] = pix[::3, ::-1]  # every third ray sampled from the deepest sample up
    scene["pixels"] = np.ascontiguousarray(pix)
    ref = run_reference_ugr(REF, scene, cuda_device)
    T._check(run_b200_ugr(scene, cuda_device), ref)


def test_ultragray_bmode_subproblem_fd64(cuda_device):
    from oracle import ultragray_oracle as UO
    from ugr_helpers import run_b200_ugr

    from us3d_b200 import scenes

    # 1,024 Gaussians of the B-mode scene that the 64 central scanlines reach, 128 samples of
    # the first 7.5 mm of depth
    sc = scenes.make_bmode_scene(1_000_000, seed=0)
    fr = scenes.bmode_sweep(64)[32]
    rays = slice(224, 288)
    x0 = float(fr.ray_origins[224, 0]) - 1.0
    x1 = float(fr.ray_origins[287, 0]) + 1.0
    z = float(fr.origin[2])
    m = sc.means
    sel = torch.nonzero((m[:, 0] > x0) & (m[:, 0] < x1) & ((m[:, 2] - z).abs() < 2.5) & (m[:, 1] < 9.0))[:, 0]
    assert sel.numel() >= 1024, sel.numel()
    gauss = sel[:1024]
    scene = _scene_dict(sc, fr, 512, 1024, 6, wr=0.0, rays=rays, samples=slice(0, 128), gauss=gauss)
    scene["grad_image"][np.abs(scene["grad_image"]) < 1e-3] = 1e-3  # no pixel in the |dL/dB| < 1e-6 skip
    out = run_b200_ugr(scene, cuda_device)
    assert out["total"] > 5000, out["total"]
    s64 = {k: (v.astype(np.float64) if isinstance(v, np.ndarray) else v) for k, v in scene.items()}
    gi = s64["grad_image"]

    def loss():
        return float((UO.render(s64, "f64")["image"] * gi).sum())

    rng = np.random.default_rng(8)
    h = 1e-4
    for key, gk in (("means", "d_means"), ("scales", "d_scales"), ("quats", "d_quats"), ("attenuations", "d_attens"),
                    ("sh", "d_sh")):
        flat = s64[key].reshape(-1)
        # parameters of Gaussians that reach some scanline (the others have zero gradient)
        live = np.nonzero(np.abs(out[gk].reshape(-1)) > 0)[0]
        picks = rng.choice(live, size=min(24, live.size), replace=False)
        fd, an = [], []
        for i in picks:
            old = flat[i]
            d = []
            for step in (h, h / 8):
                flat[i] = old + step
                lp = loss()
                flat[i] = old - step
                lm = loss()
                flat[i] = old
                d.append((lp - lm) / (2 * step))
            # a sample crossing a Gaussian's depth or echo window inside the step is a jump of
            # the loss, not a derivative: such picks (the two steps disagree) are left out
            if abs(d[0] - d[1]) > 1e-3 * max(abs(d[0]), 1e-8):
                continue
            fd.append(d[0])
            an.append(out[gk].reshape(-1)[i])
        assert len(fd) >= 16, (key, len(fd))
        e = rel_l2(np.array(an), np.array(fd))
        assert e <= 1e-4, (key, e)
