"""All five renderers on the clustered 200k-Gaussian scene and its freehand sweep, against
the reference's own CUDA builds (oracle/_ref).

Scene: 200,000 Gaussians in a 100 x 60 x 80 mm box, 20 ellipsoidal clusters plus 10 %
uniform background, log-scales N(log 0.8 mm, 0.4), opacity sigmoid(N(-1, 1)), intensity /
reflectivity U(0, 1) (us3d_b200.scenes.make_clustered_scene, seed 0). Frames: 256 x 256 px
at 0.2 mm along a random walk of 1.5 mm / 1 degree per frame (scenes.random_walk_sweep, 32
frames; four of them are rendered per renderer, all 32 for UltraGauss).

Per renderer the inputs come from the same Gaussians and probe poses:
* UltraGauss: precision factor of the scene, pixel grids of the frames;
* GaussianPile: probe-to-world pose (lateral, axial, elevational axes and origin);
* slice-adapted: the slice-adapted projection of the 3D Gaussians onto the frame (this
  library's projection, itself pinned to the reference adapter's PyTorch code by golden
  fixtures), then the bounded splat of both builds on the same 2D inputs;
* UltraGS: a pinhole camera 60 mm behind the slice along its elevational axis whose field
  of view covers the slice;
* UltraGray: one scanline per image column down the axial axis, 256 samples each.
Sort keys / sorted ids / ranges / CSR bit-exact, images <= 1e-5 and gradients <= 1e-4
relative L2 (GaussianPile scale / quaternion gradients at the reference's finite-difference
bound, see test_gaussianpile_gpu).
"""

from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
FRAMES = (0, 10, 21, 31)
H = W = 256
SPACING = 0.2


def _ref_dir(pattern):
    p = ROOT / "oracle" / "_ref"
    if not any(p.glob(pattern)):
        pytest.skip("reference build oracle/_ref not present")
    for d in (str(p), str(ROOT / "tests" / "golden")):
        if d not in sys.path:
            sys.path.insert(0, d)
    return p


@pytest.fixture(scope="module")
def config2():
    from us3d_b200 import scenes

    sc = scenes.make_clustered_scene(200_000, seed=0)
    sweep = scenes.random_walk_sweep(32, H, W, SPACING, seed=0)
    return sc, sweep


def test_config2_scene_statistics(config2):
    sc, sweep = config2
    m = sc.means.double()
    assert m.min() >= 0 and (m.max(0).values <= torch.tensor([100.0, 60.0, 80.0], dtype=torch.float64)).all()
    assert abs(float(sc.scales.double().log().mean()) - math.log(0.8)) < 0.01
    assert abs(float(torch.logit(sc.opacities.double().clamp(1e-9, 1 - 1e-9)).mean()) + 1.0) < 0.02
    steps = [float((b.origin - a.origin).norm()) for a, b in zip(sweep, sweep[1:])]
    assert max(abs(s - 1.5) for s in steps) < 1e-4


def test_config2_ultragauss(config2, cuda_device):
    _ref_dir("ultragauss_ref_C*.so")
    import test_ultragauss_gpu as T
    from ug_helpers import run_b200

    sc, sweep = config2
    g = torch.Generator().manual_seed(11)
    REF, REFK = T._reference_modules()
    for f in range(len(sweep)):
        fr = sweep[f]
        geo = np.concatenate([fr.origin.numpy(), fr.axis_lat.numpy(), fr.axis_ax.numpy(), fr.axis_ele.numpy(),
                              np.array([SPACING, SPACING, 0.0, fr.lateral_col_offset], np.float32)]).astype(np.float32)
        P = H * W
        fx = dict(means=sc.means.numpy(), precision_tril=sc.precision_tril.numpy(), opacities=sc.opacities.numpy(),
                  intensities=sc.intensities.numpy(), pixels=fr.pixels.numpy(), geo=geo, H=H, W=W,
                  chi2=np.float32(7.815), beta=np.float32(1e-4), sort_by_depth=1, bg_alpha=np.float32(1e-6),
                  bg_intensity=np.float32(0.0), d_image=torch.randn(P, generator=g).numpy(),
                  d_alpha=(0.3 * torch.randn(P, generator=g)).numpy(),
                  d_depth=(0.05 * torch.randn(P, generator=g)).numpy())
        fx.update(T._reference_run(REF, REFK, fx, cuda_device))
        T._assert_case(run_b200(fx, cuda_device), fx)


def _pose_probe_to_world(fr):
    P = torch.eye(4)
    P[:3, 0], P[:3, 1], P[:3, 2], P[:3, 3] = fr.axis_lat, fr.axis_ax, fr.axis_ele, fr.origin
    return P


def test_config2_gaussianpile(config2, cuda_device):
    _ref_dir("gaussianplie_ref_C*.so")
    import make_gaussianpile_golden as MG
    import test_gaussianpile_gpu as T
    from gp_helpers import run_b200_gp

    from oracle import gaussianpile_oracle as GO
    from ug_helpers import rel_l2

    sc, sweep = config2
    for f in FRAMES:
        fx = MG.run("config2", sc, _pose_probe_to_world(sweep[f]),
                    dict(H=H, W=W, lat=SPACING, ax=SPACING, near=0.0, centre=True, sigma_z=1.0, pose_grad=True))
        out = run_b200_gp(fx, cuda_device)
        # The pose gradient sums 200k Gaussians' contributions with lever arms of tens of mm that
        # largely cancel; the reference adds them with float atomics, this library in double in a
        # fixed order. Gradients that differ from the reference by more than 1e-4 (the pose, and
        # on some frames the means of a few very elongated footprints) are compared with the
        # FP64 oracle instead: this library must stand within 1e-4 of it or no farther than twice
        # the reference's own distance.
        m = fx["meta"].tolist()
        st = GO.render(fx["means"], fx["scales"], fx["quats"], fx["opacities"], fx["intensities"], fx["pose"],
                       fx["grid"], fx["params"], H, W, m[2], m[3], m[4], int(m[5]), m[8], precision="f64")
        g64 = GO.backward(st, fx["grad_image"], pose_grad=True)
        exact = {k: g64[k] for k in ("d_means", "d_opacity", "d_intensity", "d_pose")}
        report = {k: (rel_l2(out[k], fx["ref_" + k]), rel_l2(out[k], exact[k]), rel_l2(fx["ref_" + k], exact[k]))
                  for k in exact}
        print(f"config-2 GaussianPile frame {f}: (ours vs ref, ours vs fp64, ref vs fp64) {report}")
        T._check(out, fx, exact)


def test_config2_slice_adapted(config2, cuda_device):
    _ref_dir("slice_adapted_ref_C*.so")
    import slice_adapted_ref_bins as REFB
    import slice_adapted_ref_C as REF
    import test_slice_adapted_gpu as T
    from sa_helpers import run_b200_sa
    from us3d_b200 import slice_adapted as SA

    sc, sweep = config2
    dev = cuda_device
    t3 = [x.to(dev).contiguous() for x in (sc.means, sc.scales, sc.quats, sc.opacities.reshape(-1, 1))]
    colors = torch.stack([sc.intensities] * 3, 1).to(dev).contiguous()
    hw, hh = W * SPACING / 2, H * SPACING / 2
    g = torch.Generator().manual_seed(12)
    for f in FRAMES:
        fr = sweep[f]
        V = torch.eye(4)
        R = torch.stack([fr.axis_lat, fr.axis_ax, fr.axis_ele])  # world -> slice rotation (rows)
        centre = fr.origin + fr.axis_ax * hh  # the slice's centre: camera x lateral, y axial, z elevation
        V[:3, :3] = R
        V[:3, 3] = -(R @ centre)
        # the adapter's defaults (slice thickness 0.3 mm, cull at 3 sigma, footprint-normalised)
        st = SA.ProjectionSettings(focal_depth=0.0, slice_thickness=0.3, cull_std=3.0, thickness_scale=1.0,
                                   min_covariance=1e-4, normalize_by_footprint=True)
        # world_view_transform in the adapter's row-vector convention ([p, 1] @ view)
        m2, inv2, w2, c2, keep_idx, keep = SA.project(*t3, colors, V.t().contiguous().to(dev), st)
        m2, inv2, w2, c2 = (x.contiguous() for x in (m2, inv2, w2, c2))
        assert m2.shape[0] > 1000, m2.shape
        gi = torch.randn(H * W, 3, generator=g).to(dev)
        ga = (0.2 * torch.randn(H * W, 1, generator=g)).to(dev)
        image, alpha = REF.bounded_forward(H, W, hw, hh, m2, inv2, w2, c2, 3.0)
        dm, di, dw, dc = REF.bounded_backward(H, W, hw, hh, m2, inv2, w2, c2, gi, ga, 3.0)
        ids, starts, ends = REFB.RefTileBinning(H, W, hw, hh, m2, inv2, 3.0)
        torch.cuda.synchronize()
        c = lambda x: x.detach().cpu().numpy()  # noqa: E731
        fx = dict(H=H, W=W, half_width=np.float32(hw), half_height=np.float32(hh), radius_sigma=np.float32(3.0),
                  means2d=c(m2), inv2d=c(inv2), weights=c(w2), colors=c(c2), grad_image=c(gi), grad_alpha=c(ga),
                  ref_image=c(image), ref_alpha=c(alpha), ref_d_means=c(dm), ref_d_inv=c(di), ref_d_weights=c(dw),
                  ref_d_colors=c(dc), ref_sorted_ids=c(ids), ref_range_start=c(starts), ref_range_end=c(ends))
        T._check(run_b200_sa(fx, dev), fx, fp64_gate=True)


def test_config2_ultrags(config2, cuda_device):
    _ref_dir("ultrags_ref_C*.so")
    import test_ultrags_gpu as T
    import ultrags_ref_C as REF
    from gs_helpers import _proj, run_b200_gs, run_reference_gs

    sc, sweep = config2
    rng = np.random.default_rng(13)
    D = 60.0  # camera distance behind the slice (mm)
    for f in FRAMES:
        fr = sweep[f]
        lat, ax, ele = fr.axis_lat.double().numpy(), fr.axis_ax.double().numpy(), fr.axis_ele.double().numpy()
        centre = fr.origin.double().numpy() + ax * (H * SPACING / 2)
        cam = centre - D * ele
        Rcw = np.stack([lat, ax, ele])  # camera x = lateral, y = axial (down), z = elevation (forward)
        V = np.eye(4)
        V[:3, :3] = Rcw
        V[:3, 3] = -Rcw @ cam
        tanfovx = (W * SPACING / 2) / D
        tanfovy = (H * SPACING / 2) / D
        full = _proj(0.01, 1000.0, tanfovx, tanfovy) @ V
        fl = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
        scene = dict(means=fl(sc.means.numpy()), scales=fl(sc.scales.numpy()[:, :2]), quats=fl(sc.quats.numpy()),
                     opacities=fl(sc.opacities.numpy()[:, None]),
                     shs=fl(((sc.intensities.numpy() - 0.5) / 0.28209479177387814)[:, None, None].repeat(3, 2)),
                     colors=fl(np.zeros((0,))), transmat=fl(np.zeros((0,))), viewmatrix=fl(V.T),
                     projmatrix=fl(full.T), campos=fl(cam), bg=fl(np.zeros(3)),
                     grad_color=fl(rng.normal(size=(3, H, W))), grad_others=fl(rng.normal(size=(7, H, W))),
                     W=W, H=H, tanfovx=float(tanfovx), tanfovy=float(tanfovy), scale_modifier=1.0, sh_degree=0,
                     mode="sh")
        ref = run_reference_gs(REF, scene, cuda_device)
        out = run_b200_gs(scene, cuda_device)
        assert out["num"] > 10000, out["num"]
        T._check(out, ref, scene)


def test_config2_ultragray(config2, cuda_device):
    _ref_dir("ultragray_ref_C*.so")
    import test_ultragray_gpu as T
    import ultragray_ref_C as REF
    from ugr_helpers import run_b200_ugr, run_reference_ugr

    sc, sweep = config2
    rng = np.random.default_rng(14)
    width_mm = W * SPACING
    G = sc.means.shape[0]
    for f in FRAMES:
        fr = sweep[f]
        lat, ax, ele, o = (x.double().numpy() for x in (fr.axis_lat, fr.axis_ax, fr.axis_ele, fr.origin))
        col_off = (W - 1) * 0.5
        xs = (np.arange(W) - col_off) * (width_mm / W)
        zs = (np.arange(H) + 0.5) * SPACING
        ray_o = o[None, :] + xs[:, None] * lat[None, :]
        ray_d = np.repeat(ax[None, :], W, 0)
        pixels = ray_o[:, None, :] + zs[None, :, None] * ax[None, None, :]
        u = rng.uniform(0, 1, W)
        pert = np.arcsin(2 * u - 1) / (math.pi / 2) * 0.5
        sh = np.zeros((G, 4))
        sh[:, 0] = sc.intensities.numpy()
        fl = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
        gimg = rng.normal(size=(H, W))
        scene = dict(means=fl(sc.means.numpy()), scales=fl(sc.scales.numpy()), quats=fl(sc.quats.numpy()),
                     attenuations=fl(rng.normal(-1.0, 1.0, G)), sh=fl(sh), pixels=fl(pixels), ray_o=fl(ray_o),
                     ray_d=fl(ray_d), origin=fl(o), lat=fl(lat), ele=fl(ele), ax=fl(ax), pert=fl(pert),
                     grad_image=fl(gimg), width_mm=float(width_mm), near_mm=0.0, col_off=float(col_off),
                     elev_cut=0.0, k_sigma=3.0, wr=2.0, local=False, maxwin=17.0)
        ref = run_reference_ugr(REF, scene, cuda_device)
        out = run_b200_ugr(scene, cuda_device)
        assert out["total"] > 10000, out["total"]
        T._check(out, ref)
