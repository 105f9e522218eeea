"""Fused slice-adapted projection on the GPU against golden vectors made by the reference
adapter's PyTorch code, and the fused frame render against the reference composition
(reference projection -> reference bounded splat -> the adapter's finishing steps)."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest
import torch

from ug_helpers import rel_l2

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
NAMES = sorted(p.stem.split("_", 2)[2] for p in GOLDEN.glob("slice_projection_*.npz"))


def _load(name, dev):
    d = dict(np.load(GOLDEN / f"slice_projection_{name}.npz"))
    t = {k: torch.as_tensor(v).to(dev) for k, v in d.items() if isinstance(v, np.ndarray) and v.ndim > 0}
    return d, t


def _settings(d):
    from us3d_b200 import slice_adapted as SA

    return SA.ProjectionSettings(focal_depth=float(d["focal_depth"]), slice_thickness=float(d["set_slice_thickness_mm"]),
                                 cull_std=float(d["set_cull_std"]), thickness_scale=float(d["set_thickness_scale"]),
                                 min_covariance=float(d["set_min_covariance"]),
                                 normalize_by_footprint=bool(d["set_normalize_by_footprint"]))


@pytest.mark.parametrize("name", NAMES)
def test_fused_projection_matches_reference_golden(name, cuda_device):
    from us3d_b200 import slice_adapted as SA

    d, t = _load(name, cuda_device)
    s = _settings(d)
    m2, inv, w, col, idx, mask = SA.project(t["means"], t["scales"], t["quats"], t["opacities"], t["colors"], t["view"], s)
    np.testing.assert_array_equal(mask.cpu().numpy(), d["ref_keep"])
    np.testing.assert_array_equal(idx.cpu().numpy(), np.nonzero(d["ref_keep"])[0])
    for k, v in (("means2d", m2), ("inv2d", inv), ("weights", w), ("colors", col)):
        assert rel_l2(v.cpu().numpy(), d["ref_" + k]) <= 1e-5, (k, rel_l2(v.cpu().numpy(), d["ref_" + k]))
    g = SA.project_backward(idx, t["means"], t["scales"], t["quats"], t["opacities"], t["view"], s, t["up_means2d"],
                            t["up_inv2d"], t["up_weights"], t["up_colors"])
    for k, v in zip(("means", "scales", "quats", "opacities", "colors"), g):
        r = d["ref_d_" + k]
        assert rel_l2(v.cpu().numpy().reshape(r.shape), r) <= 1e-4, (k, rel_l2(v.cpu().numpy().reshape(r.shape), r))


def _camera(d, dev, H=120, W=160):
    from slice_adapted_3dgs_renderer.fused import SliceCameraInput

    return SliceCameraInput(image_height=H, image_width=W, half_width_mm=16.0, half_height_mm=12.0,
                            focal_depth_mm=float(d["focal_depth"]), world_view_transform=torch.as_tensor(d["view"]).to(dev))


def _render_settings(d, **kw):
    from slice_adapted_3dgs_renderer.fused import SliceAdaptedRenderSettings

    return SliceAdaptedRenderSettings(slice_thickness_mm=float(d["set_slice_thickness_mm"]),
                                      cull_std=float(d["set_cull_std"]), thickness_scale=float(d["set_thickness_scale"]),
                                      min_covariance=float(d["set_min_covariance"]),
                                      normalize_by_footprint=bool(d["set_normalize_by_footprint"]), **kw)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("gray", [True, False])
def test_fused_render_matches_reference_composition(name, gray, cuda_device):
    from slice_adapted_3dgs_renderer.fused import SliceAdapted3DGSInput, render_slice_adapted_3dgs

    p = ROOT / "oracle" / "_ref"
    if not any(p.glob("slice_adapted_ref_C*.so")):
        pytest.skip("reference build not present")
    sys.path.insert(0, str(p))
    import slice_adapted_ref_C as REF

    d, t = _load(name, cuda_device)
    cam = _camera(d, cuda_device)
    st = _render_settings(d, bg_color=0.05, output_grayscale=gray)
    out = render_slice_adapted_3dgs(SliceAdapted3DGSInput(t["means"], t["scales"], t["quats"], t["opacities"],
                                                          t["colors"]), cam, st)
    # reference composition: its projection (golden) -> its bounded splat -> adapter finishing (render.py:100-129)
    img, alpha = REF.bounded_forward(cam.image_height, cam.image_width, cam.half_width_mm, cam.half_height_mm,
                                     t["ref_means2d"].contiguous(), t["ref_inv2d"].contiguous(),
                                     t["ref_weights"].contiguous(), t["ref_colors"].contiguous(), st.cull_std)
    img = (img + st.bg_color).clamp(0.0, 1.0).transpose(0, 1).reshape(3, cam.image_height, cam.image_width)
    alpha = alpha.transpose(0, 1).reshape(1, cam.image_height, cam.image_width)
    if gray:
        img = (0.299 * img[0] + 0.587 * img[1] + 0.114 * img[2]).unsqueeze(0)
    assert rel_l2(out.image.cpu().numpy(), img.cpu().numpy()) <= 2e-5
    assert rel_l2(out.extras["alpha_image"].cpu().numpy(), alpha.cpu().numpy()) <= 2e-5
    np.testing.assert_array_equal(out.extras["visibility_filter"].cpu().numpy(), d["ref_keep"])


@pytest.mark.parametrize("name", NAMES)
def test_fused_render_autograd_chain(name, cuda_device):
    """Gradients of the fused render equal the projection VJP applied to the bounded splat's
    gradients of the kept splats (both parity-tested on their own)."""
    from slice_adapted_3dgs_renderer import additive_splat_bounded
    from slice_adapted_3dgs_renderer.fused import SliceAdapted3DGSInput, render_slice_adapted_3dgs
    from us3d_b200 import slice_adapted as SA

    d, t = _load(name, cuda_device)
    cam = _camera(d, cuda_device)
    st = _render_settings(d, clamp_output=False, output_grayscale=False)
    leaves = [t[k].clone().requires_grad_(True) for k in ("means", "scales", "quats", "opacities", "colors")]
    out = render_slice_adapted_3dgs(SliceAdapted3DGSInput(*leaves), cam, st)
    up = torch.randn(out.image.shape, generator=torch.Generator(device=cuda_device).manual_seed(7),
                     device=cuda_device)
    (out.image * up).sum().backward()
    s = _settings(d)
    m2, inv, w, col, idx, _ = SA.project(t["means"], t["scales"], t["quats"], t["opacities"], t["colors"], t["view"], s)
    ps = [x.clone().requires_grad_(True) for x in (m2, inv, w, col)]
    img, _ = additive_splat_bounded(cam.image_height, cam.image_width, cam.half_width_mm, cam.half_height_mm, *ps,
                                    st.cull_std)
    (img.transpose(0, 1).reshape(3, cam.image_height, cam.image_width) * up).sum().backward()
    g = SA.project_backward(idx, t["means"], t["scales"], t["quats"], t["opacities"], t["view"], s,
                            *[p_.grad for p_ in ps])
    for leaf, ref in zip(leaves, g):
        np.testing.assert_allclose(leaf.grad.cpu().numpy().reshape(-1), ref.cpu().numpy().reshape(-1), rtol=1e-5,
                                   atol=1e-7)
