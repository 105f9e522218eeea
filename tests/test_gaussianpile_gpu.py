"""GaussianPile parity on the GPU through the C ABI: against golden fixtures from the
reference's own CUDA build, the live reference build, and the C oracle.

Tolerances: tile rectangles, sorted ids and tile ranges bit-exact; images <= 1e-5
relative L2; mean / opacity / intensity / pose gradients <= 1e-4 relative L2 against the
reference backward. Scale and quaternion gradients are, as in the reference, central
differences (step 1e-3) of an adjoint-weighted footprint in fp32; they are compared at
<= 1e-3 relative L2, because the reference's own float-atomic accumulation order changes
the adjoint in its last bits and the finite difference amplifies that.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest
import torch

from gp_helpers import gp_golden_names, load_gp, run_b200_gp
from ug_helpers import rel_l2

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def _check(out, fx, exact=None):
    """Binning bit-exact, image <= 1e-5 and gradients <= 1e-4 against the reference. With
    ``exact`` (the FP64 oracle's gradients of the same inputs), a gradient further than 1e-4
    from the reference passes when it stands no farther from the FP64 values than 1e-4 or twice
    the reference's own distance from them: on large scenes a few very elongated footprints
    (conditional covariance entries in the hundreds) amplify fp32 rounding in both
    implementations, each in its own summation order."""
    vis = fx["ref_rects"][:, 0] < fx["ref_rects"][:, 2]
    np.testing.assert_array_equal(out["rects"][vis], fx["ref_rects"][vis], err_msg="tile rectangles")
    np.testing.assert_array_equal(out["sorted_ids"], fx["ref_sorted_ids"], err_msg="sorted ids")
    np.testing.assert_array_equal(out["range_start"], fx["ref_range_start"], err_msg="range start")
    np.testing.assert_array_equal(out["range_end"], fx["ref_range_end"], err_msg="range end")
    assert rel_l2(out["image"], fx["ref_image"]) <= 1e-5, rel_l2(out["image"], fx["ref_image"])
    names = ("d_means", "d_opacity", "d_intensity") + (("d_pose",) if int(fx["pose_grad"]) else ())
    for k in names:
        e = rel_l2(out[k], fx["ref_" + k])
        if e <= 1e-4:
            continue
        assert exact is not None, (k, e)
        ours, ref = rel_l2(out[k], exact[k]), rel_l2(fx["ref_" + k], exact[k])
        assert ours <= max(1e-4, 2.0 * ref), (k, e, ours, ref)
    for k in ("d_scales", "d_quats"):
        assert rel_l2(out[k], fx["ref_" + k]) <= 1e-3, (k, rel_l2(out[k], fx["ref_" + k]))


@pytest.mark.parametrize("name", gp_golden_names() or ["c1"])
def test_gaussianpile_golden_parity(name, cuda_device):
    fx = load_gp(name)
    _check(run_b200_gp(fx, cuda_device), fx)


def test_gaussianpile_live_reference(cuda_device):
    p = ROOT / "oracle" / "_ref"
    if not any(p.glob("gaussianplie_ref_C*.so")):
        pytest.skip("reference build not present")
    sys.path.insert(0, str(p))
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    import make_gaussianpile_golden as MG

    from us3d_b200 import scenes

    sc = scenes.make_scene(20000, seed=9, cube_mm=60.0, opacity_mu=-1.0)
    fx = MG.run("live", sc, MG.pose_matrix(3.0, (0.2, 1, 0), (30.0, 5.0, 30.0)),
                dict(H=256, W=256, lat=0.2, ax=0.2, near=0.0, centre=True, sigma_z=1.0, pose_grad=True))
    _check(run_b200_gp(fx, cuda_device), fx)


def test_gaussianpile_oracle_agreement(cuda_device):
    from oracle import gaussianpile_oracle as GO

    fx = load_gp("c1")
    out = run_b200_gp(fx, cuda_device)
    m = fx["meta"].tolist()
    st = GO.render(fx["means"], fx["scales"], fx["quats"], fx["opacities"], fx["intensities"], fx["pose"], fx["grid"],
                   fx["params"], int(fx["H"]), int(fx["W"]), m[2], m[3], m[4], int(m[5]), m[8])
    np.testing.assert_array_equal(st["sorted_ids"], out["sorted_ids"])
    assert rel_l2(out["image"], st["image"]) <= 1e-5
    g = GO.backward(st, fx["grad_image"], pose_grad=True)
    for k in ("d_means", "d_opacity"):
        assert rel_l2(out[k], g[k]) <= 1e-4, (k, rel_l2(out[k], g[k]))
    # The pose gradient is a sum over all Gaussians with heavy cancellation; the CPU
    # restatement (IEEE division/exp, no FMA) and the fast-math GPU build differ by a few
    # 1e-4 there. Against the reference's own GPU build it agrees to 1e-4 (golden tests).
    assert rel_l2(out["d_pose"], g["d_pose"]) <= 2e-3


def test_gaussianpile_dropin_api(cuda_device):
    """GaussianPlieRenderer through autograd equals the low-level path; pose gradient only
    when the pose requires grad."""
    from types import SimpleNamespace

    from gaussianplie_renderer import GaussianPlieRenderConfig, GaussianPlieRenderer, build_slice_grid_pack

    fx = load_gp("c1")
    dev = cuda_device
    cfg = GaussianPlieRenderConfig(H=int(fx["H"]), W=int(fx["W"]), lateral_spacing_mm_per_pix=0.3,
                                   axial_spacing_mm_per_pix=0.3, axial_near_mm=0.0, sigma_z_mm=1.0)
    r = GaussianPlieRenderer(cfg)
    r.set_slice_grid_geometry(build_slice_grid_pack(SimpleNamespace(H=cfg.H, W=cfg.W, delta_lateral_mm=0.3,
                                                                    delta_axial_mm=0.3, near_mm=0.0,
                                                                    center_lateral=True), dev))
    T = lambda k: torch.as_tensor(fx[k]).to(dev).requires_grad_(True)  # noqa: E731
    means, scales, quats, alphas = T("means"), T("scales"), T("quats"), T("opacities")
    pose = torch.as_tensor(fx["pose"]).to(dev).requires_grad_(True)
    img = r(means, scales, quats, alphas, pose)
    assert img.shape == (cfg.H, cfg.W)
    (img * torch.as_tensor(fx["grad_image"]).to(dev)).sum().backward()
    assert rel_l2(img.detach().cpu().numpy(), fx["ref_image"]) <= 1e-5
    assert rel_l2(means.grad.cpu().numpy(), fx["ref_d_means"]) <= 1e-4
    assert rel_l2(pose.grad.cpu().numpy(), fx["ref_d_pose"]) <= 1e-4


@pytest.mark.parametrize("tile", [7, 12, 32])
def test_gaussianpile_tile_sizes_same_image(tile, cuda_device):
    """Tile lists hold candidates in Gaussian order whatever the tile size, and each pixel
    applies the same box and weight tests, so the image does not depend on tile_size_px
    (including sizes whose blocks end in a partial warp)."""
    fx = load_gp((gp_golden_names() or ["c1"])[0])
    from us3d_b200 import gaussianpile as GP

    dev = cuda_device
    t = lambda k: torch.as_tensor(fx[k]).to(dev).float().contiguous()  # noqa: E731
    m = fx["meta"].tolist()
    args = (t("means"), t("scales"), t("quats"), t("opacities").reshape(-1), t("intensities").reshape(-1),
            t("pose").reshape(16), t("grid"), t("params"), int(fx["H"]), int(fx["W"]), m[2], m[3], m[4])
    ref, _ = GP.forward(*args, 16, m[8], bool(m[9]))
    img, _ = GP.forward(*args, tile, m[8], bool(m[9]))
    assert torch.equal(img, ref)


def _gp_case(G, seed, H, W, spacing, sigma_z, radius_sigma, cube_mm, log_scale_mean, device):
    """Inputs of a small projected-slice case (the values the drop-in renderer sends)."""
    from types import SimpleNamespace

    from gaussianplie_renderer import GaussianPlieRenderConfig, build_slice_grid_pack
    from gaussianplie_renderer.autograd import _meta_vector, _us_focus_params_vector
    from us3d_b200 import scenes

    sc = scenes.make_scene(G, seed=seed, cube_mm=cube_mm, log_scale_mean=log_scale_mean, opacity_mu=-0.5)
    # weight threshold 1e-12 (the reference's floor): a pixel whose weight crosses it jumps by
    # less than 1e-12, so finite differences see no cut there
    cfg = GaussianPlieRenderConfig(H=H, W=W, lateral_spacing_mm_per_pix=spacing, axial_spacing_mm_per_pix=spacing,
                                   axial_near_mm=0.0, sigma_z_mm=sigma_z, radius_sigma=radius_sigma,
                                   opacity_cull_threshold=1e-12)
    grid = build_slice_grid_pack(SimpleNamespace(H=H, W=W, delta_lateral_mm=spacing, delta_axial_mm=spacing,
                                                 near_mm=0.0, center_lateral=True), device)
    # probe->world pose: slice through the cube centre, turned a little about two axes
    a, b = 0.21, -0.13
    Rx = torch.tensor([[1, 0, 0], [0, np.cos(a), -np.sin(a)], [0, np.sin(a), np.cos(a)]], dtype=torch.float64)
    Ry = torch.tensor([[np.cos(b), 0, np.sin(b)], [0, 1, 0], [-np.sin(b), 0, np.cos(b)]], dtype=torch.float64)
    R = Rx @ Ry
    pose = torch.eye(4, dtype=torch.float64)
    pose[:3, :3] = R
    pose[:3, 3] = torch.tensor([cube_mm / 2] * 3, dtype=torch.float64) - R[:, 1] * (H * spacing / 2)
    meta = _meta_vector(cfg, device).cpu().numpy()
    params = _us_focus_params_vector(cfg, device)
    g = torch.Generator().manual_seed(seed + 5)
    return dict(means=sc.means.numpy(), scales=sc.scales.numpy(), quats=sc.quats.numpy(),
                opacities=sc.opacities.numpy(), intensities=np.ones(G, np.float32), pose=pose.float().numpy(),
                grid=grid.cpu().numpy(), params=params.cpu().numpy(), meta=meta, H=H, W=W,
                grad_image=torch.randn((H, W), generator=g).numpy())


def _gp_gpu(fx, device, mode):
    from us3d_b200 import gaussianpile as GP

    t = lambda k: torch.as_tensor(fx[k]).to(device).float().contiguous()  # noqa: E731
    m = fx["meta"].tolist()
    img, b = GP.forward(t("means"), t("scales"), t("quats"), t("opacities").reshape(-1), t("intensities").reshape(-1),
                        t("pose").reshape(16), t("grid"), t("params"), int(fx["H"]), int(fx["W"]), m[2], m[3], m[4],
                        int(m[5]), m[8], bool(m[9]))
    grads = GP.backward(b, t("grad_image"), True, shape_gradients=mode)
    torch.cuda.synchronize()
    return img.cpu().numpy(), [x.cpu().numpy() for x in grads]


def test_gaussianpile_analytic_gradients_fd64(cuda_device):
    """The analytic shape adjoint (and every other gradient) of the GPU backward against
    central finite differences (step 1e-4) of the FP64 oracle's image, on a small scene with
    a wide cut-off (radius_sigma 8: the box and weight thresholds change the image by less
    than 1e-13), <= 1e-4 relative L2 over the sampled parameters.

    The pose gradient: the reference differentiates the slice covariance a_i^T Sigma_w a_j
    with respect to the axes as if Sigma_w were symmetric (Sigma_w a_j and Sigma_w a_i), but
    its Sigma_w = R D R is symmetric only when R is. Its translation entries are exact for any
    scene and are checked here; the nine axis entries are checked on the same scene with every
    quaternion turned into a half turn (w = 0, R = 2uu^T - I, symmetric), where the
    reference's formula is the derivative. On other scenes they are compared with the
    reference itself (the config-2 and golden tests)."""
    from oracle import gaussianpile_oracle as GO

    fx = _gp_case(48, 21, 40, 48, 0.5, 1.2, 8.0, 20.0, float(np.log(1.6)), cuda_device)
    img, (dm, ds, dq, do, di, dp) = _gp_gpu(fx, cuda_device, "analytic")
    m = fx["meta"].tolist()
    w = fx["grad_image"].astype(np.float64).reshape(-1)

    def loss(means, scales, quats, opac, pose):
        st = GO.render(means, scales, quats, opac, fx["intensities"].astype(np.float64), pose, fx["grid"], fx["params"],
                       int(fx["H"]), int(fx["W"]), m[2], m[3], m[4], int(m[5]), m[8], precision="f64")
        return float(np.dot(w, st["image"].reshape(-1)))

    base = [fx[k].astype(np.float64).copy() for k in ("means", "scales", "quats", "opacities", "pose")]
    st0 = GO.render(*base[:4], fx["intensities"], base[4], fx["grid"], fx["params"], int(fx["H"]), int(fx["W"]), m[2],
                    m[3], m[4], int(m[5]), m[8], precision="f64")
    assert rel_l2(img, st0["image"]) <= 1e-5
    rng = np.random.default_rng(3)
    h = 1e-4
    for which, (name, an) in enumerate(zip(("d_means", "d_scales", "d_quats", "d_opacity", "d_pose"),
                                           (dm, ds, dq, do, dp))):
        arr = base[which]
        idx = rng.choice(arr.size, size=min(24, arr.size), replace=False) if which < 4 else np.array([3, 7, 11])
        fd = []
        for fi in idx:
            plus = [b.copy() for b in base]
            minus = [b.copy() for b in base]
            plus[which].reshape(-1)[fi] += h
            minus[which].reshape(-1)[fi] -= h
            fd.append((loss(*plus) - loss(*minus)) / (2 * h))
        e = rel_l2(an.reshape(-1)[idx], np.array(fd))
        assert e <= 1e-4, (name, e)

    # half turns: the full 3x4 pose block against finite differences
    q = fx["quats"].astype(np.float64)
    u = q[:, 1:] / np.linalg.norm(q[:, 1:], axis=1, keepdims=True)
    fx_h = dict(fx, quats=np.concatenate([np.zeros((q.shape[0], 1)), u], 1).astype(np.float32))
    _, (*_g, dp_h) = _gp_gpu(fx_h, cuda_device, "analytic")
    base_h = [fx_h[k].astype(np.float64).copy() for k in ("means", "scales", "quats", "opacities", "pose")]
    fd = []
    for fi in range(12):
        plus = [b.copy() for b in base_h]
        minus = [b.copy() for b in base_h]
        plus[4].reshape(-1)[fi] += h
        minus[4].reshape(-1)[fi] -= h
        fd.append((loss(*plus) - loss(*minus)) / (2 * h))
    e = rel_l2(dp_h.reshape(-1)[:12], np.array(fd))
    assert e <= 1e-4, ("d_pose, half turns", e)


def test_gaussianpile_shape_gradients_reference_floor(cuda_device):
    """The reference's scale / quaternion gradients are central differences (step 1e-3) in
    fp32 of an adjoint that it sums with float atomics. Run twice on one input they differ (the
    run-to-run floor, measured here: a few 1e-5 to 1e-4), and they stand far from the exact
    derivative (the analytic mode, itself checked against FP64 finite differences): the fp32
    difference quotient loses most digits where a Gaussian's footprint barely depends on its
    shape (nearly isotropic Gaussians and quaternions). The finite-difference mode here evaluates
    the same quotient on this library's deterministic adjoint; it agrees with the reference to
    <= 1e-3, a few times the reference's own spread and far inside the quotient's distance from
    the derivative, which the test also bounds."""
    p = ROOT / "oracle" / "_ref"
    if not any(p.glob("gaussianplie_ref_C*.so")):
        pytest.skip("reference build not present")
    sys.path.insert(0, str(p))
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    import make_gaussianpile_golden as MG

    from us3d_b200 import scenes

    sc = scenes.make_scene(20000, seed=9, cube_mm=60.0, opacity_mu=-1.0)
    args = (sc, MG.pose_matrix(3.0, (0.2, 1, 0), (30.0, 5.0, 30.0)),
            dict(H=256, W=256, lat=0.2, ax=0.2, near=0.0, centre=True, sigma_z=1.0, pose_grad=True))
    r1 = MG.run("a", *args)
    r2 = MG.run("b", *args)
    out = run_b200_gp(r1, cuda_device)
    _, (_, ds_an, dq_an, *_rest) = _gp_gpu(r1, cuda_device, "analytic")
    report = {}
    for k, an in (("d_scales", ds_an), ("d_quats", dq_an)):
        floor = rel_l2(r2["ref_" + k], r1["ref_" + k])
        ours = rel_l2(out[k], r1["ref_" + k])
        report[k] = dict(floor=floor, ours_fd=ours, ref_vs_analytic=rel_l2(r1["ref_" + k], an),
                         ours_fd_vs_analytic=rel_l2(out[k], an))
    print("gaussianpile shape-gradient floor:", report)
    for k, r in report.items():
        assert r["ours_fd"] <= 1e-3, (k, r)
        assert r["ours_fd"] <= 0.05 * r["ref_vs_analytic"], (k, r)
