"""UltraGauss parity on the GPU, through the C ABI (ctypes) of libus3d_b200.so.

Checks against (1) golden fixtures produced by the reference's own CUDA build,
(2) the reference build run live (oracle/_ref, when present), (3) the C oracle, and
(4) FP64 central finite differences. Tolerances (from the workload specification):
sort keys, tile ranges and per-pixel candidate counts/lists bit-exact; images <= 1e-5
relative L2; gradients <= 1e-4 relative L2 against the reference backward.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest
import torch

from ug_helpers import golden_names, load_golden, rel_l2, run_b200

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
IMG_TOL = 1e-5
GRAD_TOL = 1e-4


def _assert_case(out, fx, prefix="ref_"):
    np.testing.assert_array_equal(out["keys"], fx[prefix + "keys"].astype(np.int64), err_msg="sorted keys")
    np.testing.assert_array_equal(out["values"], fx[prefix + "values"], err_msg="sorted values")
    np.testing.assert_array_equal(out["range_start"], fx[prefix + "range_start"], err_msg="range start")
    np.testing.assert_array_equal(out["range_end"], fx[prefix + "range_end"], err_msg="range end")
    np.testing.assert_array_equal(out["counts"], fx[prefix + "counts"], err_msg="pixel candidate counts")
    np.testing.assert_array_equal(out["offsets"], fx[prefix + "offsets"], err_msg="pixel offsets")
    np.testing.assert_array_equal(out["indices"], fx[prefix + "indices"], err_msg="pixel candidate indices")
    for k in ("image", "alpha", "depth"):
        assert rel_l2(out[k], fx[prefix + k]) <= IMG_TOL, (k, rel_l2(out[k], fx[prefix + k]))
    for k in ("d_means", "d_tril", "d_opacity", "d_intensity"):
        assert rel_l2(out[k], fx[prefix + k]) <= GRAD_TOL, (k, rel_l2(out[k], fx[prefix + k]))


@pytest.mark.parametrize("name", golden_names() or ["c1"])
def test_golden_reference_parity(name, cuda_device):
    fx = load_golden(name)
    out = run_b200(fx, cuda_device)
    _assert_case(out, fx)


def _reference_modules():
    p = ROOT / "oracle" / "_ref"
    if not any(p.glob("ultragauss_ref_C*.so")):
        pytest.skip("reference build oracle/_ref not present")
    sys.path.insert(0, str(p))
    import ultragauss_ref_C
    import ultragauss_ref_keys

    return ultragauss_ref_C, ultragauss_ref_keys


def _reference_run(REF, REFK, fx, device):
    dev = device
    t = lambda k: torch.as_tensor(fx[k]).to(dev).contiguous()  # noqa: E731
    pad = lambda x: torch.nn.functional.pad(x, (0, 1)).contiguous()  # noqa: E731
    geo = torch.as_tensor(fx["geo"]).to(dev)
    o, l, a, e = geo[0:3].contiguous(), geo[3:6].contiguous(), geo[6:9].contiguous(), geo[9:12].contiguous()
    H, W = int(fx["H"]), int(fx["W"])
    dlat, dax, near, coloff = (float(x) for x in fx["geo"][12:16])
    chi2, beta, sort = float(fx["chi2"]), float(fx["beta"]), bool(fx["sort_by_depth"])
    mp, pp, tril = pad(t("means")), pad(t("pixels")), t("precision_tril")
    counts, offsets, indices = REF.MapperForwardCUDA(pp, mp, tril, o, l, a, e, H, W, dlat, dax, near, coloff, chi2,
                                                     sort, beta)
    attr = torch.stack([t("opacities"), t("intensities")], 1).contiguous()
    image, alpha, depth, sic = REF.ShaderForwardCUDA(attr, mp, tril, pp, o, e, offsets, counts, indices,
                                                     float(fx["bg_alpha"]), float(fx["bg_intensity"]), chi2, beta)
    dm, dt, da = REF.ShaderBackwardCUDA(t("d_image"), t("d_alpha"), t("d_depth"), attr, mp, tril, pp, o, e, offsets,
                                        counts, indices, sic, alpha, float(fx["bg_alpha"]), float(fx["bg_intensity"]),
                                        chi2, beta)
    _, _, _, keys, vals, rs, re = REFK.RefBinning(mp, tril, o, l, a, e, H, W, dlat, dax, near, coloff, chi2, sort, beta)
    torch.cuda.synchronize()
    c = lambda x: x.detach().cpu().numpy()  # noqa: E731
    return dict(ref_keys=c(keys), ref_values=c(vals), ref_range_start=c(rs), ref_range_end=c(re), ref_counts=c(counts),
                ref_offsets=c(offsets), ref_indices=c(indices), ref_image=c(image), ref_alpha=c(alpha),
                ref_depth=c(depth), ref_d_means=c(dm)[:, :3], ref_d_tril=c(dt), ref_d_opacity=c(da)[:, 0],
                ref_d_intensity=c(da)[:, 1])


def _scene_case(G, H, W, spacing, seed, frame=0, n_frames=4, sort=True, bg_a=1e-6, bg_i=0.0, chi2=7.815, beta=1e-4,
                **kw):
    from us3d_b200 import scenes

    sc = scenes.make_scene(G, seed=seed, **kw)
    fr = scenes.linear_sweep(n_frames, H, W, spacing, seed=seed, cube_mm=kw.get("cube_mm", 64.0))[frame]
    g = torch.Generator().manual_seed(seed + 7)
    P = H * W
    geo = np.concatenate([fr.origin.numpy(), fr.axis_lat.numpy(), fr.axis_ax.numpy(), fr.axis_ele.numpy(),
                          np.array([spacing, spacing, 0.0, fr.lateral_col_offset], np.float32)]).astype(np.float32)
    return dict(means=sc.means.numpy(), precision_tril=sc.precision_tril.numpy(), opacities=sc.opacities.numpy(),
                intensities=sc.intensities.numpy(), pixels=fr.pixels.numpy(), geo=geo, H=H, W=W,
                chi2=np.float32(chi2), beta=np.float32(beta), sort_by_depth=int(sort), bg_alpha=np.float32(bg_a),
                bg_intensity=np.float32(bg_i), d_image=torch.randn(P, generator=g).numpy(),
                d_alpha=(0.3 * torch.randn(P, generator=g)).numpy(), d_depth=(0.05 * torch.randn(P, generator=g)).numpy())


@pytest.mark.parametrize(
    "G,H,W,spacing,seed,sort",
    [(4096, 128, 128, 0.3, 0, True), (20000, 256, 256, 0.25, 1, True), (3000, 100, 60, 0.5, 2, False),
     (60000, 192, 320, 0.2, 3, True)],
)
def test_live_reference_parity(G, H, W, spacing, seed, sort, cuda_device):
    REF, REFK = _reference_modules()
    fx = _scene_case(G, H, W, spacing, seed, frame=1, sort=sort)
    fx.update(_reference_run(REF, REFK, fx, cuda_device))
    out = run_b200(fx, cuda_device)
    _assert_case(out, fx)


def test_live_reference_parity_dense_tiles(cuda_device):
    """120000 Gaussians in a 16 mm cube under a 96x96 slice: tile buckets of every size class
    of the tile sort (in-register segments, the 48 KB shared-memory pass, the 64 KB packed pass
    for 4097-8192 keys, the 192 KB pass up to 16384, the global-memory network above) against
    the reference's own binning."""
    REF, REFK = _reference_modules()
    fx = _scene_case(120000, 96, 96, 0.25, 5, frame=1, cube_mm=16.0)
    fx.update(_reference_run(REF, REFK, fx, cuda_device))
    n = fx["ref_range_end"] - fx["ref_range_start"]
    print("bucket sizes: max", int(n.max()), "in (4096, 8192]:", int(((n > 4096) & (n <= 8192)).sum()),
          "in (8192, 16384]:", int(((n > 8192) & (n <= 16384)).sum()))
    assert n.max() > 16384 and ((n > 64) & (n <= 2048)).any()
    assert ((n > 4096) & (n <= 8192)).any() and ((n > 8192) & (n <= 16384)).any()
    out = run_b200(fx, cuda_device)
    _assert_case(out, fx)


def test_live_reference_parity_many_gaussians(cuda_device):
    """More Gaussians than the tile sort packs into one 64-bit word (2^20 - 1): the shared-memory
    pass sorts keys with their slot payload; keys, ranges, candidate lists, image and gradients
    against the reference's own build."""
    REF, REFK = _reference_modules()
    fx = _scene_case(1100000, 96, 80, 0.25, 13, frame=1)
    fx.update(_reference_run(REF, REFK, fx, cuda_device))
    out = run_b200(fx, cuda_device)
    _assert_case(out, fx)


@pytest.mark.parametrize("beta", [1e-12, 5e-11])
def test_live_reference_parity_windowed(beta, cuda_device):
    """A diagonal offset in (0, 1e-10) (the reference's clamp inside the window radii can then
    cut the chi-square ellipsoid): the kernels that apply the lateral/axial window per pair, against
    the reference's own binning, candidate lists, forward and backward."""
    REF, REFK = _reference_modules()
    fx = _scene_case(20000, 160, 128, 0.25, 11, frame=2, beta=beta)
    fx.update(_reference_run(REF, REFK, fx, cuda_device))
    out = run_b200(fx, cuda_device)
    _assert_case(out, fx)


def test_oracle_agreement(cuda_device):
    """GPU vs the C oracle (IEEE CPU arithmetic): counts differ at most by the oracle's
    near-threshold window tests; image and gradients within tolerance."""
    from oracle import ultragauss_oracle as O

    fx = _scene_case(8192, 128, 160, 0.3, 5, frame=2)
    out = run_b200(fx, cuda_device)
    st = O.render(fx["means"], fx["precision_tril"], fx["opacities"], fx["intensities"], fx["pixels"], fx["geo"],
                  int(fx["H"]), int(fx["W"]), float(fx["chi2"]), float(fx["beta"]), True, float(fx["bg_alpha"]),
                  float(fx["bg_intensity"]))
    assert np.all(np.abs(out["counts"] - st["counts"]) <= st["ambiguous"])
    assert rel_l2(out["image"], st["image"]) <= IMG_TOL
    g = O.backward(st, fx["d_image"], fx["d_alpha"], fx["d_depth"])
    for k in ("d_means", "d_tril", "d_opacity", "d_intensity"):
        assert rel_l2(out[k], g[k]) <= GRAD_TOL, (k, rel_l2(out[k], g[k]))


def test_fd_gradients_fp64(cuda_device):
    """Central finite differences (step 1e-4) of the FP64 oracle forward vs the GPU
    adjoint, on a small scene with a wide chi-square window so no pair crosses a cut."""
    from oracle import ultragauss_oracle as O

    fx = _scene_case(48, 32, 32, 0.6, 11, frame=1, n_frames=3, chi2=400.0, cube_mm=19.2, log_scale_mean=0.7,
                     bg_a=1e-3)
    fx["intensities"] = (0.1 + 0.8 * fx["intensities"]).astype(np.float32)
    out = run_b200(fx, cuda_device)
    wI, wA, wD = fx["d_image"].astype(np.float64), fx["d_alpha"].astype(np.float64), fx["d_depth"].astype(np.float64)

    def loss(means, tril, op, it):
        st = O.render(means, tril, op, it, fx["pixels"].astype(np.float64), fx["geo"].astype(np.float64),
                      int(fx["H"]), int(fx["W"]), float(fx["chi2"]), float(fx["beta"]), True, float(fx["bg_alpha"]),
                      float(fx["bg_intensity"]), precision="f64", want_indices=True, want_ambiguous=False)
        return float(np.dot(wI, st["image"]) + np.dot(wA, st["alpha"]) + np.dot(wD, st["depth"]))

    base = [fx[k].astype(np.float64).copy() for k in ("means", "precision_tril", "opacities", "intensities")]
    rng = np.random.default_rng(0)
    h = 1e-4
    fd, an = [], []
    for which, key in enumerate(("d_means", "d_tril", "d_opacity", "d_intensity")):
        arr = base[which]
        flat_idx = rng.choice(arr.size, size=min(24, arr.size), replace=False)
        for fi in flat_idx:
            plus = [b.copy() for b in base]
            minus = [b.copy() for b in base]
            plus[which].reshape(-1)[fi] += h
            minus[which].reshape(-1)[fi] -= h
            fd.append((loss(*plus) - loss(*minus)) / (2 * h))
            an.append(out[key].reshape(-1)[fi])
    err = rel_l2(an, fd)
    print(f"FD gradient check (FP64 oracle, h=1e-4): rel-L2 {err:.3e} over {len(fd)} entries")
    assert err <= 2e-3, err


def test_batched_frames_match_single(cuda_device):
    """Many frames of different sizes binned and shaded in one launch sequence give each
    frame's single-frame result; gradients are the sum over frames."""
    from us3d_b200 import scenes
    from us3d_b200 import ultragauss as UG

    dev = cuda_device
    sc = scenes.make_scene(30000, seed=4).to(dev)
    sizes = [(128, 128, 0.5), (96, 200, 0.32), (256, 256, 0.25), (50, 70, 0.9)]
    specs, pix, grads = [], [], []
    g = torch.Generator().manual_seed(3)
    for i, (H, W, s) in enumerate(sizes):
        fr = scenes.linear_sweep(len(sizes), H, W, s, seed=4)[i]
        specs.append(UG.SliceSpec(H, W, s, s, 0.0, fr.lateral_col_offset, fr.origin, fr.axis_lat, fr.axis_ax,
                                  fr.axis_ele))
        pix.append(fr.pixels)
        grads.append(torch.randn(3, H * W, generator=g))
    args = (sc.means, sc.precision_tril.contiguous(), sc.opacities, sc.intensities)
    ft = UG.build_frame_table(specs, dev)
    allpix = torch.cat(pix).to(dev)
    b = UG.bin_gaussians(*args, ft, 7.815, 1e-4, True)
    img, alp, dep, cnt = UG.forward(b, allpix, 1e-6, 0.0)
    gg = torch.cat(grads, dim=1).to(dev)
    dsum = UG.backward(b, allpix, gg[0].contiguous(), gg[1].contiguous(), gg[2].contiguous(), alp, 1e-6, 0.0)
    acc = [torch.zeros_like(x) for x in dsum]
    off = 0
    for i, sp in enumerate(specs):
        n = sp.height * sp.width
        f1 = UG.build_frame_table([sp], dev)
        b1 = UG.bin_gaussians(*args, f1, 7.815, 1e-4, True)
        i1, a1, d1, c1 = UG.forward(b1, pix[i].to(dev), 1e-6, 0.0)
        assert torch.equal(i1, img[off:off + n]) and torch.equal(c1, cnt[off:off + n])
        assert torch.equal(a1, alp[off:off + n]) and torch.equal(d1, dep[off:off + n])
        gi = grads[i].to(dev)
        d = UG.backward(b1, pix[i].to(dev), gi[0].contiguous(), gi[1].contiguous(), gi[2].contiguous(), a1, 1e-6, 0.0)
        for a_, d_ in zip(acc, d):
            a_ += d_
        off += n
    for a_, d_ in zip(acc, dsum):
        assert rel_l2(d_.cpu().numpy(), a_.cpu().numpy()) <= 1e-5


def test_backward_deterministic(cuda_device):
    fx = _scene_case(20000, 128, 128, 0.4, 6)
    a = run_b200(fx, cuda_device)
    b = run_b200(fx, cuda_device)
    for k in ("d_means", "d_tril", "d_opacity", "d_intensity", "image"):
        assert np.array_equal(a[k], b[k]), k


def test_capacity_retry_and_oversized_tile(cuda_device):
    """A capacity far below the instance count is grown and re-binned; a tile holding more
    instances than the in-shared-memory sort takes the global-memory path, same result."""
    from oracle import ultragauss_oracle as O

    from us3d_b200 import scenes

    fx = _scene_case(12000, 16, 16, 0.05, 8, log_scale_mean=-1.0)
    geo = np.array([0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 1, 0.05, 0.05, 0.0, 0.0], np.float32)
    fx["geo"] = geo
    fx["pixels"] = scenes.slice_pixels(torch.zeros(3), torch.tensor([1.0, 0, 0]), torch.tensor([0, 1.0, 0]), 16, 16,
                                       0.05, 0.05, 0.0, 0.0).numpy()
    rng = np.random.default_rng(0)
    fx["means"] = (np.array([0.4, 0.4, 0.0]) + rng.normal(0, 0.05, (12000, 3))).astype(np.float32)
    out = run_b200(fx, cuda_device, capacity=16)
    st = O.render(fx["means"], fx["precision_tril"], fx["opacities"], fx["intensities"], fx["pixels"], fx["geo"],
                  16, 16, float(fx["chi2"]), float(fx["beta"]), True, float(fx["bg_alpha"]), 0.0)
    assert out["keys"].shape[0] > 8192
    same = np.mean(out["keys"] == st["keys"].astype(np.int64))
    assert same > 0.999, same
    assert rel_l2(out["image"], st["image"]) <= IMG_TOL


def test_empty_and_invalid_inputs(cuda_device):
    from ultragauss_renderer import SliceGeometry, UltraGaussRenderConfig, UltraGaussRenderer

    dev = cuda_device
    cfg = UltraGaussRenderConfig(H=20, W=33, lateral_spacing_mm_per_pix=0.5, axial_spacing_mm_per_pix=0.5,
                                 axial_near_mm=0.0, fixed_bg_alpha=0.2, fixed_bg_intensity=0.4)
    geom = SliceGeometry(torch.zeros(3, device=dev), torch.tensor([1.0, 0, 0], device=dev),
                         torch.tensor([0, 1.0, 0], device=dev), torch.tensor([0, 0, 1.0], device=dev))
    pix = torch.rand(20 * 33, 3, device=dev)
    z = torch.zeros((0, 3), device=dev)
    img, alpha, depth, inter = UltraGaussRenderer(cfg)(z, torch.zeros((0, 6), device=dev), torch.zeros(0, device=dev),
                                                       torch.zeros(0, device=dev), pix, geom, True)
    assert torch.allclose(img, torch.full_like(img, 0.4)) and torch.allclose(alpha, torch.full_like(alpha, 0.2))
    assert int(inter["pixel_gauss_counts"].sum()) == 0 and inter["pixel_gauss_indices"].numel() == 0
    with pytest.raises(RuntimeError, match="n_pixels must equal H\\*W"):
        UltraGaussRenderer(cfg)(z, torch.zeros((0, 6), device=dev), torch.zeros(0, device=dev),
                                torch.zeros(0, device=dev), pix[:-1], geom)


def test_dropin_autograd_matches_lowlevel(cuda_device):
    from ultragauss_renderer import SliceGeometry, UltraGaussRenderConfig, UltraGaussRenderer

    fx = _scene_case(5000, 96, 128, 0.4, 9, bg_a=1e-6)
    low = run_b200(fx, cuda_device)
    dev = cuda_device
    geo = fx["geo"]
    cfg = UltraGaussRenderConfig(H=96, W=128, lateral_spacing_mm_per_pix=0.4, axial_spacing_mm_per_pix=0.4,
                                 axial_near_mm=0.0, lateral_col_offset=float(geo[15]), fixed_bg_alpha=1e-6)
    T = lambda k: torch.as_tensor(fx[k]).to(dev).requires_grad_(True)  # noqa: E731
    means, tril, op, it = T("means"), T("precision_tril"), T("opacities"), T("intensities")
    g = lambda a, b: torch.as_tensor(geo[a:b]).to(dev)  # noqa: E731
    img, alpha, depth, inter = UltraGaussRenderer(cfg)(means, tril, op, it, torch.as_tensor(fx["pixels"]).to(dev),
                                                       SliceGeometry(g(0, 3), g(3, 6), g(6, 9), g(9, 12)), True)
    assert not inter.is_materialized("pixel_gauss_indices")
    loss = ((img.reshape(-1) * torch.as_tensor(fx["d_image"]).to(dev)).sum()
            + (alpha.reshape(-1) * torch.as_tensor(fx["d_alpha"]).to(dev)).sum()
            + (depth.reshape(-1) * torch.as_tensor(fx["d_depth"]).to(dev)).sum())
    loss.backward()
    assert np.array_equal(img.detach().cpu().numpy().reshape(-1), low["image"])
    assert np.array_equal(inter["pixel_gauss_indices"].cpu().numpy(), low["indices"])
    assert np.array_equal(inter["pixel_gauss_offsets"].cpu().numpy(), low["offsets"])
    for p, k in ((means, "d_means"), (tril, "d_tril"), (op, "d_opacity"), (it, "d_intensity")):
        assert rel_l2(p.grad.cpu().numpy(), low[k]) <= 1e-6, k


def _cull_case(dev, G=120000, sizes=((256, 256, 0.125), (200, 330, 0.2), (128, 96, 0.4)), jitter=0.0, seed=8,
               scale_mm=1.0):
    from us3d_b200 import scenes
    from us3d_b200 import ultragauss as UG

    sc = scenes.make_scene(G, seed=seed, log_scale_mean=float(np.log(scale_mm))).to(dev)
    specs, pix, grads = [], [], []
    g = torch.Generator().manual_seed(seed)
    for i, (H, W, s) in enumerate(sizes):
        fr = scenes.linear_sweep(len(sizes), H, W, s, seed=seed)[i]
        specs.append(UG.SliceSpec(H, W, s, s, fr.axial_near, fr.lateral_col_offset, fr.origin, fr.axis_lat,
                                  fr.axis_ax, fr.axis_ele))
        p = fr.pixels.clone()
        if jitter > 0:
            p += jitter * torch.randn(p.shape, generator=g)
        pix.append(p)
        grads.append(torch.randn(3, H * W, generator=g))
    args = (sc.means, sc.precision_tril.contiguous(), sc.opacities, sc.intensities)
    return args, UG.build_frame_table(specs, dev), torch.cat(pix).to(dev), torch.cat(grads, dim=1).to(dev)


def test_culled_batched_deterministic(cuda_device):
    """Slice-culled batched binning + forward + backward, three times, each on device memory
    that held random bytes just before (freed to the caching allocator, so the workspace
    reuses it): images and gradients are bit-identical, i.e. nothing reads memory that the
    step did not write and no result depends on the order of atomic updates."""
    from us3d_b200 import ultragauss as UG

    args, ft, pix, grads = _cull_case(cuda_device, G=200000)
    runs = []
    for r in range(3):
        junk = torch.randint(0, 256, (int(3e8),), dtype=torch.uint8, device=cuda_device)
        del junk
        b = UG.bin_gaussians(*args, ft, 7.815, 1e-4, True, slice_cull_pixels=pix)
        img, alpha, depth, _ = UG.forward(b, pix, 1e-6, 0.0, want_counts=False)
        g = UG.backward(b, pix, grads[0], grads[1], grads[2], alpha, 1e-6, 0.0)
        runs.append([x.cpu().numpy() for x in (img, alpha, depth, *g)])
    for r in runs[1:]:
        for x, y in zip(runs[0], r):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("jitter,scale,beta", [(0.0, 1.0, 1e-4), (0.0, 0.3, 1e-4), (2e-3, 1.0, 1e-4), (0.5, 1.0, 1e-4),
                                               (0.0, 1.0, 1e-12)])
def test_slice_cull_identical_results(jitter, scale, beta, cuda_device):
    """A slice-culled binning keeps fewer instances but gives bit-identical images, alpha,
    depth and gradients (pixels on the frame grid, slightly off it, and far off it; beta below
    1e-10 runs the kernels that apply the window per pair)."""
    from us3d_b200 import ultragauss as UG

    args, ft, pix, gg = _cull_case(cuda_device, jitter=jitter, scale_mm=scale)
    out = {}
    for cull in (False, True):
        b = UG.bin_gaussians(*args, ft, 7.815, beta, True, slice_cull_pixels=pix if cull else None)
        img, alp, dep, cnt = UG.forward(b, pix, 1e-6, 0.0)
        assert (cnt is None) == cull
        d = UG.backward(b, pix, gg[0].contiguous(), gg[1].contiguous(), gg[2].contiguous(), alp, 1e-6, 0.0)
        out[cull] = (b.total, img, alp, dep) + tuple(d)
    assert out[True][0] <= out[False][0]
    if jitter < 0.1:
        assert out[True][0] < 0.9 * out[False][0], (out[True][0], out[False][0])
    for a, c in zip(out[False][1:], out[True][1:]):
        assert torch.equal(a, c)


def test_slice_cull_dropin_renderer(cuda_device):
    from ultragauss_renderer import SliceGeometry, UltraGaussRenderConfig, UltraGaussRenderer
    from us3d_b200 import scenes

    dev = cuda_device
    sc = scenes.make_scene(40000, seed=9).to(dev)
    fr = scenes.linear_sweep(3, 160, 160, 0.25, seed=9)[1].to(dev)
    cfg = UltraGaussRenderConfig(H=160, W=160, lateral_spacing_mm_per_pix=0.25, axial_spacing_mm_per_pix=0.25,
                                 axial_near_mm=fr.axial_near, lateral_col_offset=fr.lateral_col_offset)
    geo = SliceGeometry(fr.origin, fr.axis_lat, fr.axis_ax, fr.axis_ele)
    res = []
    for inter in (True, False):
        ps = [x.clone().requires_grad_(True) for x in (sc.means, sc.precision_tril, sc.opacities, sc.intensities)]
        img, alpha, depth, _ = UltraGaussRenderer(cfg)(*ps, fr.pixels, geo, return_intermediates=inter)
        (img.square().sum() + alpha.sum() + depth.sum()).backward()
        res.append([img.detach(), alpha.detach(), depth.detach()] + [p.grad for p in ps])
    for a, c in zip(*res):
        assert torch.equal(a, c)


def test_autograd_steps_free_memory_without_gc(cuda_device):
    """Forward + backward through both autograd entry points (the drop-in renderer and the
    batched renderer), with the cyclic garbage collector off: once a step's tensors are dropped,
    the memory in use returns to its level before the step (nothing the step allocated is kept
    alive by a reference cycle through the autograd graph)."""
    import gc

    from ultragauss_renderer import SliceGeometry, UltraGaussRenderConfig, UltraGaussRenderer
    from us3d_b200 import scenes
    from us3d_b200 import ultragauss as UG
    from us3d_b200.batch import UltraGaussBatchRenderer

    dev = cuda_device
    sc = scenes.make_scene(40000, seed=9).to(dev)
    sweep = scenes.linear_sweep(3, 160, 160, 0.25, seed=9)
    fr = sweep[1].to(dev)
    cfg = UltraGaussRenderConfig(H=160, W=160, lateral_spacing_mm_per_pix=0.25, axial_spacing_mm_per_pix=0.25,
                                 axial_near_mm=fr.axial_near, lateral_col_offset=fr.lateral_col_offset)
    geo = SliceGeometry(fr.origin, fr.axis_lat, fr.axis_ax, fr.axis_ele)
    specs = [UG.SliceSpec(f.height, f.width, f.lateral_spacing, f.axial_spacing, f.axial_near, f.lateral_col_offset,
                          f.origin, f.axis_lat, f.axis_ax, f.axis_ele) for f in sweep]
    batch_pix = torch.cat([f.pixels for f in sweep]).to(dev)
    batched = UltraGaussBatchRenderer(specs, dev)

    def dropin_step():
        ps = [x.clone().requires_grad_(True) for x in (sc.means, sc.precision_tril, sc.opacities, sc.intensities)]
        img, alpha, depth, _ = UltraGaussRenderer(cfg)(*ps, fr.pixels, geo, return_intermediates=False)
        (img.sum() + alpha.sum() + depth.sum()).backward()

    def batched_step():
        ps = [x.clone().requires_grad_(True) for x in (sc.means, sc.precision_tril, sc.opacities, sc.intensities)]
        img, alpha, depth = batched(*ps, batch_pix)
        (img.sum() + alpha.sum() + depth.sum()).backward()
        batched.last = {}

    gc.collect()
    was_enabled = gc.isenabled()
    gc.disable()
    try:
        for step in (dropin_step, batched_step):
            step()  # first call: kernel attributes, cached backward scratch
            torch.cuda.synchronize()
            before = torch.cuda.memory_allocated(dev)
            for _ in range(3):
                step()
            torch.cuda.synchronize()
            assert torch.cuda.memory_allocated(dev) == before, step.__name__
    finally:
        if was_enabled:
            gc.enable()


def test_graphed_training_step_matches_eager(cuda_device):
    """A CUDA-graph replay of bin + forward + loss gradient + backward equals the same step
    run eagerly, also after the parameters are updated in place between replays."""
    from us3d_b200 import ultragauss as UG
    from us3d_b200.batch import GraphedTrainingStep

    dev = cuda_device
    args, ft, pix, gg = _cull_case(dev, G=60000, sizes=((128, 128, 0.25), (96, 160, 0.3)))
    params = [a.clone() for a in args]
    tgt = torch.rand(pix.shape[0], generator=torch.Generator().manual_seed(1)).to(dev)

    def loss_grad(img, alpha, depth):
        return torch.sign(img - tgt) / img.numel(), 0.1 * alpha, torch.zeros_like(depth)

    from us3d_b200 import scenes

    sizes = ((128, 128, 0.25), (96, 160, 0.3))
    specs = []
    for i, (H, W, s) in enumerate(sizes):
        fr = scenes.linear_sweep(len(sizes), H, W, s, seed=8)[i]
        specs.append(UG.SliceSpec(H, W, s, s, fr.axial_near, fr.lateral_col_offset, fr.origin, fr.axis_lat,
                                  fr.axis_ax, fr.axis_ele))
    step = GraphedTrainingStep(specs, dev, params, pix, loss_grad)

    def eager():
        b = UG.bin_gaussians(*params, ft, 7.815, 1e-4, True)
        img, alpha, depth, _ = UG.forward(b, pix, 1e-6, 0.0)
        dI, dA, dD = loss_grad(img, alpha, depth)
        return UG.backward(b, pix, dI, dA, dD, alpha, 1e-6, 0.0)

    for it in range(2):
        got = [x.clone() for x in step.replay()]
        step.check()
        ref = eager()
        for a_, b_ in zip(got, ref):
            assert torch.equal(a_, b_), it
        params[0].add_(0.01)  # in-place update seen by the next replay


def test_launch_shapes_same_results_and_autotune(cuda_device):
    """Every launch shape of the shading kernels (forward batch 128/256/512, backward CTA
    128/256 threads) and both forward variants (one pixel per thread, two pixels per thread in
    packed f32x2) give bit-identical images and gradients for each backward variant; the two
    backward variants (scalar FP32, packed f32x2 pairs) give the same images and gradients
    within summation-order rounding; the autotuner times every (shape, variant pair) and keeps
    the fastest."""
    from ug_helpers import rel_l2
    from us3d_b200 import batch as B
    from us3d_b200 import ultragauss as UG

    args, ft, pix, grads = _cull_case(cuda_device, G=60000)
    default = B.get_launch_config()
    default_variant = B.get_backward_variant()
    default_fvariant = B.get_forward_variant()
    outs = {}
    try:
        for fvariant in B.FORWARD_VARIANTS:
            B.set_forward_variant(fvariant)
            for variant in B.BACKWARD_VARIANTS:
                B.set_backward_variant(variant)
                for shape in B.LAUNCH_SHAPES:
                    B.set_launch_config(*shape)
                    b = UG.bin_gaussians(*args, ft, 7.815, 1e-4, True, slice_cull_pixels=pix)
                    img, alpha, depth, _ = UG.forward(b, pix, 1e-6, 0.0, want_counts=False)
                    g = UG.backward(b, pix, grads[0], grads[1], grads[2], alpha, 1e-6, 0.0)
                    outs[(*shape, variant, fvariant)] = [x.cpu().numpy() for x in (img, alpha, depth, *g)]
        for variant in B.BACKWARD_VARIANTS:
            ref = outs[(*default, variant, 0)]
            for fvariant in B.FORWARD_VARIANTS:
                for shape in B.LAUNCH_SHAPES:
                    for x, y in zip(outs[(*shape, variant, fvariant)], ref):
                        assert np.array_equal(x, y), (shape, variant, fvariant)
        scalar, packed = outs[(*default, 0, 0)], outs[(*default, 1, 0)]
        for x, y in zip(scalar[:3], packed[:3]):
            assert np.array_equal(x, y)  # the forward is the same kernel
        for x, y in zip(scalar[3:], packed[3:]):
            assert rel_l2(y, x) <= 1e-5
        timings = B.autotune_launch(ft, list(args), pix, reps=1)
        assert set(timings) == {(*s, v, f) for s in B.LAUNCH_SHAPES for v in B.BACKWARD_VARIANTS
                                for f in B.FORWARD_VARIANTS if not (f == 1 and s[0] == 512)}
        best = min(timings, key=timings.get)
        assert B.get_launch_config() == best[:2] and B.get_backward_variant() == best[2]
        assert B.get_forward_variant() == best[3]
    finally:
        B.set_launch_config(*default)
        B.set_backward_variant(default_variant)
        B.set_forward_variant(default_fvariant)
