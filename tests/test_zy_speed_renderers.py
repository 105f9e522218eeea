"""Throughput of the reference's own CUDA (built for sm_100a by oracle/build_ref.py) next to
this library for the four other renderers, forward + backward on the same inputs and the same
B200: GaussianPile (projected-slice us_focus), slice-adapted 3DGS (bounded additive splat),
UltraGS (2D-Gaussian surfels) and UltraGray (scanline transmission). Sizes follow the
survey's config 2 (200k Gaussians, 256x256 frames) unless US3D_SPEED_SCALE (a float factor on
the Gaussian counts) says otherwise. Results are printed (pytest -s) and each test asserts that
the library is faster than the reference."""

from __future__ import annotations

import os
import sys
from pathlib import Path

import pytest
import torch

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
SCALE = float(os.environ.get("US3D_SPEED_SCALE", "1.0"))


def _ref(name):
    p = ROOT / "oracle" / "_ref"
    if not any(p.glob(f"{name}*.so")):
        pytest.skip("reference build not present")
    for q in (str(p), str(ROOT / "tests" / "golden")):
        if q not in sys.path:
            sys.path.insert(0, q)
    return __import__(name)


def _time(fn, reps, trials=5):
    """Median over ``trials`` of the mean CUDA-event time of ``reps`` calls, after three
    warm-up calls (the first calls size workspaces and caches; a trial that catches a clock
    ramp or another process's burst does not decide the figure)."""
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = []
    for _ in range(trials):
        st.record()
        for _ in range(reps):
            fn()
        en.record()
        torch.cuda.synchronize()
        out.append(st.elapsed_time(en) / reps)
    return sorted(out)[len(out) // 2]


def _report(name, what, ms_ref, ms_ours):
    print(f"\n[speed] {name}: {what}\n[speed]   reference CUDA (sm_100a build) {ms_ref:9.3f} ms/frame"
          f"\n[speed]   this library                   {ms_ours:9.3f} ms/frame   speed-up {ms_ref / ms_ours:.1f}x")
    assert ms_ours < ms_ref


def test_speed_gaussianpile(cuda_device):
    REF = _ref("gaussianplie_ref_C")
    import make_gaussianpile_golden as MG

    from gaussianplie_renderer import GaussianPlieRenderConfig, build_slice_grid_pack
    from gaussianplie_renderer.autograd import _meta_vector, _us_focus_params_vector
    from types import SimpleNamespace

    from us3d_b200 import gaussianpile as GP
    from us3d_b200 import scenes

    dev = cuda_device
    G, H, W = int(200000 * SCALE), 256, 256
    sc = scenes.make_scene(G, seed=9, cube_mm=60.0, opacity_mu=-1.0)
    pose = MG.pose_matrix(3.0, (0.2, 1, 0), (30.0, 5.0, 30.0)).to(dev).contiguous()
    cfg = GaussianPlieRenderConfig(H=H, W=W, lateral_spacing_mm_per_pix=0.2, axial_spacing_mm_per_pix=0.2,
                                   axial_near_mm=0.0, sigma_z_mm=1.0)
    grid = build_slice_grid_pack(SimpleNamespace(H=H, W=W, delta_lateral_mm=0.2, delta_axial_mm=0.2, near_mm=0.0,
                                                 center_lateral=True), dev)
    meta = _meta_vector(cfg, dev)
    params = _us_focus_params_vector(cfg, dev)
    m = meta.cpu().tolist()
    t = [x.to(dev).float().contiguous() for x in (sc.means, sc.scales, sc.quats, sc.opacities, torch.ones(G))]
    grad = torch.randn((H, W), generator=torch.Generator().manual_seed(7)).to(dev).reshape(-1).contiguous()

    def ref_step():
        colors, rects, ids, rs, re = REF.ProjectedSliceForwardCUDA(
            *t, pose, grid, params, H, W, m[2], m[3], m[4], int(m[5]), m[6], m[7], m[8], int(m[10]), int(m[11]),
            int(m[12]), bool(m[9]), int(m[13]), m[14], int(m[15]))
        REF.ProjectedSliceBackwardCUDA(*t, pose, grid, params, rects, 0, H, W, int(m[5]), m[2], m[3], m[4], m[8],
                                       int(m[13]), m[14], int(m[10]), ids, rs, re, grad, int(m[15]), True)

    def ours_step():
        img, b = GP.forward(*t, pose.reshape(16), grid, params, H, W, m[2], m[3], m[4], int(m[5]), m[8], bool(m[9]))
        GP.backward(b, grad.reshape(H, W), True)

    _report("GaussianPile", f"{G} Gaussians, {H}x{W} slice, fwd+bwd incl. pose gradient", _time(ref_step, 3),
            _time(ours_step, 5))


def test_speed_slice_adapted(cuda_device):
    REF = _ref("slice_adapted_ref_C")
    import make_slice_adapted_golden as MG

    from us3d_b200 import slice_adapted as SA

    dev = cuda_device
    N, H, W, hw, hh = int(100000 * SCALE), 256, 256, 25.6, 25.6
    means, inv, weights, colors, gi, ga = [x.to(dev) for x in MG.make_inputs(N, H, W, hw, hh, 3)]

    def ref_step():
        REF.bounded_forward(H, W, hw, hh, means, inv, weights, colors, 3.0)
        REF.bounded_backward(H, W, hw, hh, means, inv, weights, colors, gi, ga, 3.0)

    def ours_step():
        image, alpha, b = SA.bounded_forward(H, W, hw, hh, means, inv, weights, colors, 3.0)
        SA.bounded_backward(b, hw, hh, means, inv, weights, colors, gi, ga, 3.0)

    _report("slice-adapted 3DGS", f"{N} projected Gaussians, {H}x{W}, bounded splat fwd+bwd", _time(ref_step, 3),
            _time(ours_step, 5))


def test_speed_ultrags(cuda_device):
    REF = _ref("ultrags_ref_C")
    import gs_helpers as GH

    from us3d_b200 import surfel as S

    dev = cuda_device
    P, H, W = int(200000 * SCALE), 256, 256
    scene = GH.make_scene(P, W, H, 4)
    t = GH._args(scene, dev)
    op = t["opacities"]

    def ref_step():
        num, color, others, radii, gb, bb, ib = REF.rasterize_gaussians(
            t["bg"], t["means"], t["colors"], op, t["scales"], t["quats"], scene["scale_modifier"], t["transmat"],
            t["viewmatrix"], t["projmatrix"], scene["tanfovx"], scene["tanfovy"], H, W, t["shs"], scene["sh_degree"],
            t["campos"], False, False)
        REF.rasterize_gaussians_backward(
            t["bg"], t["means"], radii, t["colors"], t["scales"], t["quats"], scene["scale_modifier"], t["transmat"],
            t["viewmatrix"], t["projmatrix"], scene["tanfovx"], scene["tanfovy"], t["grad_color"], t["grad_others"],
            t["shs"], scene["sh_degree"], t["campos"], gb, num, bb, ib, False)

    def ours_step():
        num, color, others, radii, state = S.forward(t["bg"], t["means"], t["colors"], op.reshape(-1), t["scales"],
                                                      t["quats"], scene["scale_modifier"], t["transmat"],
                                                      t["viewmatrix"], t["projmatrix"], H, W, t["shs"],
                                                      scene["sh_degree"], t["campos"], False)
        S.backward(state, t["bg"], t["means"], radii, t["colors"], t["scales"], t["quats"], scene["scale_modifier"],
                   t["transmat"], t["viewmatrix"], t["projmatrix"], scene["tanfovx"], scene["tanfovy"],
                   t["grad_color"], t["grad_others"], t["shs"], scene["sh_degree"], t["campos"])

    _report("UltraGS", f"{P} surfels, {H}x{W}, colour + 7 auxiliary maps, fwd+bwd", _time(ref_step, 3),
            _time(ours_step, 5))


def test_speed_ultragray(cuda_device):
    REF = _ref("ultragray_ref_C")
    import torch.nn.functional as F
    import ugr_helpers as UH

    from us3d_b200 import ultragray as U

    dev = cuda_device
    G, W, H = int(100000 * SCALE), 128, 512
    scene = UH.make_scene(G, W, H, 5)
    t = {k: torch.as_tensor(scene[k]).to(dev).contiguous() for k in UH.SCENE_ARRAYS}
    mp = F.pad(t["means"], (0, 1)).contiguous()
    sp = F.pad(t["scales"], (0, 1)).contiguous()
    p = UH.params(scene)

    def ref_step():
        counts, offsets, idx, depths = REF.MapperForwardCUDA(mp, sp, t["origin"], t["lat"], t["ele"], t["ax"], W,
                                                             scene["width_mm"], scene["near_mm"], scene["col_off"],
                                                             scene["elev_cut"], scene["k_sigma"])
        args = (mp, sp, t["quats"], t["attenuations"], t["sh"], counts, offsets, idx, depths, t["pixels"],
                t["ray_o"], t["ray_d"], t["ele"], t["pert"], scene["k_sigma"], scene["wr"], bool(scene["local"]),
                scene["maxwin"])
        REF.ShaderForwardCUDA(*args)
        REF.ShaderBackwardCUDA(t["grad_image"], *args)

    def ours_step():
        image, b = U.forward(t["means"], t["scales"], t["quats"], t["attenuations"], t["sh"], t["pixels"], t["ray_o"],
                             t["ray_d"], t["origin"], t["lat"], t["ele"], t["ax"], t["pert"], p)
        U.backward(b, t["quats"], t["pixels"], t["ray_o"], t["ray_d"], t["ele"], t["pert"], t["grad_image"], p)

    _report("UltraGray", f"{G} Gaussians, {W} scanlines x {H} samples, fwd+bwd", _time(ref_step, 1),
            _time(ours_step, 3))
