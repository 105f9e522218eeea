"""The training step around the UltraGauss renderer on the GPU: the per-frame loss and its
gradient coefficients against PyTorch autograd of the reference's image_loss (L1 + global
SSIM, pipeline_god_file.py:606-637), the multi-tensor Adam launch against torch.optim.Adam
(with the logistic activation's chain rule), the fused-loss backward against the unfused one,
and whole training steps of UltraGaussTrainer against the reference's PyTorch training loop
(GaussianParameters activations + drop-in renderer + image_loss + torch.optim.Adam)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def rel(a: torch.Tensor, b: torch.Tensor) -> float:
    a, b = a.double().reshape(-1), b.double().reshape(-1)
    return float((a - b).norm() / b.norm().clamp_min(1e-30))


def _simple_ssim(x, y):
    c1, c2 = 0.01 ** 2, 0.03 ** 2
    mux, muy = x.mean(), y.mean()
    vx = ((x - mux) ** 2).mean()
    vy = ((y - muy) ** 2).mean()
    vxy = ((x - mux) * (y - muy)).mean()
    return ((2 * mux * muy + c1) * (2 * vxy + c2)) / ((mux ** 2 + muy ** 2 + c1) * (vx + vy + c2))


def _image_loss(x, y, w1, ws):
    total = w1 * torch.mean(torch.abs(x - y))
    if ws > 0:
        total = total + ws * (1.0 - _simple_ssim(x, y))
    return total


def _specs(sizes, seed=3, cube_mm=32.0):
    from us3d_b200 import scenes
    from us3d_b200 import ultragauss as UG

    out, pix = [], []
    for i, (H, W, s) in enumerate(sizes):
        fr = scenes.linear_sweep(len(sizes), H, W, s, seed=seed, cube_mm=cube_mm)[i]
        out.append(UG.SliceSpec(H, W, s, s, fr.axial_near, fr.lateral_col_offset, fr.origin, fr.axis_lat, fr.axis_ax,
                                fr.axis_ele))
        pix.append(fr.pixels)
    return out, torch.cat(pix)


@pytest.mark.parametrize("w1,ws", [(1.0, 0.0), (1.0, 0.2), (0.5, 1.0)])
def test_loss_and_gradient_coefficients(w1, ws, cuda_device):
    from us3d_b200 import ultragauss as UG

    dev = cuda_device
    sizes = ((64, 80, 0.3), (33, 47, 0.5), (128, 128, 0.2))
    specs, _ = _specs(sizes)
    ft = UG.build_frame_table(specs, dev)
    g = torch.Generator().manual_seed(5)
    P = sum(h * w for h, w, _ in sizes)
    x = torch.rand(P, generator=g).to(dev)
    y = torch.rand(P, generator=g).to(dev)
    x[:7] = y[:7]  # ties: sign(0) = 0 as torch.abs' gradient
    stats, coef = UG.loss(ft, x, y, w1, ws)
    off = 0
    for f, (H, W, _) in enumerate(sizes):
        n = H * W
        xd = x[off:off + n].double().requires_grad_(True)
        yd = y[off:off + n].double()
        # the weights reach the kernels as float32
        L = _image_loss(xd, yd, float(np.float32(w1)), float(np.float32(ws)))
        L.backward()
        st = stats[f].cpu()
        lv = float(L.detach())
        assert abs(float(st[7]) - lv) <= 1e-9 * max(1.0, abs(lv)), (f, float(st[7]), lv)
        assert abs(float(st[6]) - float(_simple_ssim(xd.detach(), yd))) <= 1e-9
        k = coef[f]
        xs, ys = x[off:off + n], y[off:off + n]
        grad = k[0] * torch.sign(xs - ys) + k[1] + k[2] * xs + k[3] * ys
        assert rel(grad, xd.grad) <= 2e-6, (f, rel(grad, xd.grad))
        off += n


def test_adam_matches_torch(cuda_device):
    from us3d_b200.train import Adam

    dev = cuda_device
    g = torch.Generator().manual_seed(11)
    shapes = [(1000, 3), (777, 6), (1000, 1), (5,)]
    logistic = [False, False, True, False]
    ours = [torch.randn(s, generator=g).to(dev) for s in shapes]
    ref = [torch.nn.Parameter(p.clone()) for p in ours]
    opt_ref = torch.optim.Adam(ref, lr=1e-2, betas=(0.9, 0.999), eps=1e-8)
    opt = Adam(ours, lr=1e-2, betas=(0.9, 0.999), eps=1e-8, logistic=logistic)
    for step in range(5):
        grads = [torch.randn(s, generator=g).to(dev) * (10.0 ** (step - 2)) for s in shapes]
        opt_ref.zero_grad(set_to_none=True)
        for p, gr, lg in zip(ref, grads, logistic):
            out = torch.sigmoid(p) if lg else p
            out.backward(gr)
        opt_ref.step()
        opt.step([gr.contiguous() for gr in grads])
    for a, b in zip(ours, ref):
        assert rel(a, b.detach()) <= 1e-6, rel(a, b.detach())


def _scene(dev, G=20000, seed=4):
    from us3d_b200 import scenes

    sc = scenes.make_scene(G, seed=seed, cube_mm=32.0)
    return sc


def test_backward_loss_matches_unfused(cuda_device):
    from us3d_b200 import ultragauss as UG

    dev = cuda_device
    sc = _scene(dev)
    specs, pix = _specs(((96, 128, 0.25), (80, 80, 0.3)), seed=4)
    pix = pix.to(dev)
    ft = UG.build_frame_table(specs, dev)
    args = (sc.means.to(dev), sc.precision_tril.to(dev).contiguous(), sc.opacities.to(dev), sc.intensities.to(dev))
    b = UG.bin_gaussians(*args, ft, 7.815, 1e-4, True, slice_cull_pixels=pix)
    img, alpha, depth, _ = UG.forward(b, pix, 1e-6, 0.0, want_counts=False)
    tgt = torch.rand(img.shape, generator=torch.Generator().manual_seed(2)).to(dev)
    stats, coef = UG.loss(ft, img, tgt, 1.0, 0.3)
    fused = UG.backward_loss(b, pix, img, tgt, coef, alpha, 1e-6, 0.0)
    dI = torch.empty_like(img)
    off = 0
    for f, sp in enumerate(specs):
        n = sp.height * sp.width
        k = coef[f]
        xs, ys = img[off:off + n], tgt[off:off + n]
        dI[off:off + n] = k[0] * torch.sign(xs - ys) + k[1] + k[2] * xs + k[3] * ys
        off += n
    z = torch.zeros_like(img)
    unfused = UG.backward(b, pix, dI, z, z, alpha, 1e-6, 0.0)
    for a, c in zip(fused, unfused):
        assert rel(a, c) <= 1e-6, rel(a, c)


def _torch_pipeline_steps(params0, specs, pix, tgts, cfg, steps, dev):
    """The reference's training loop for UltraGauss, with this repository's drop-in renderer:
    nn.Parameters, sigmoid activations, image_loss per frame (summed over the batch), Adam."""
    from ultragauss_renderer import SliceGeometry, UltraGaussRenderConfig, UltraGaussRenderer

    ps = [torch.nn.Parameter(t.clone()) for t in params0]
    opt = torch.optim.Adam(ps, lr=cfg.lr, betas=(cfg.beta1, cfg.beta2), eps=cfg.eps)
    for _ in range(steps):
        opt.zero_grad(set_to_none=True)
        means, tril, raw_o, raw_i = ps
        total = 0.0
        off = 0
        for sp, in_pix, tgt in zip(specs, pix, tgts):
            rc = UltraGaussRenderConfig(H=sp.height, W=sp.width, lateral_spacing_mm_per_pix=sp.lateral_spacing,
                                        axial_spacing_mm_per_pix=sp.axial_spacing, axial_near_mm=sp.axial_near,
                                        lateral_col_offset=sp.lateral_col_offset, chi2_threshold=cfg.chi2_threshold,
                                        mapper_sort_by_depth=cfg.sort_by_depth, diag_beta=cfg.diag_beta,
                                        fixed_bg_alpha=cfg.bg_alpha, fixed_bg_intensity=cfg.bg_intensity)
            geom = SliceGeometry(sp.origin.to(dev), sp.axis_lat.to(dev), sp.axis_ax.to(dev), sp.axis_ele.to(dev))
            img, _, _, _ = UltraGaussRenderer(rc)(means, tril, torch.sigmoid(raw_o).reshape(-1),
                                                  torch.sigmoid(raw_i).reshape(-1), in_pix, geom, False)
            total = total + _image_loss(img.reshape(-1), tgt, cfg.l1_weight, cfg.ssim_weight)
        total.backward()
        opt.step()
    return [p.detach() for p in ps]


@pytest.mark.parametrize("ssim_weight,graph", [(0.0, True), (0.25, True), (0.25, False)])
def test_trainer_matches_torch_training_loop(ssim_weight, graph, cuda_device):
    from us3d_b200 import scenes
    from us3d_b200.train import TrainConfig, UltraGaussParameters, UltraGaussTrainer

    dev = cuda_device
    sizes = ((96, 128, 0.25), (80, 80, 0.3))
    specs, pix = _specs(sizes, seed=4)
    pix = pix.to(dev)
    sc = scenes.make_scene(20000, seed=4, cube_mm=32.0)
    params = UltraGaussParameters.from_points(sc.means.to(dev), sc.intensities.to(dev), init_scale_mm=0.8)
    g = torch.Generator().manual_seed(9)
    tgt = torch.rand(pix.shape[0], generator=g).to(dev)
    cfg = TrainConfig(lr=1e-2, ssim_weight=ssim_weight)
    start = [t.clone() for t in params.tensors()]
    trainer = UltraGaussTrainer(params, [(specs, pix, tgt)], cfg, graph=graph)
    steps = 3
    for _ in range(steps):
        trainer.step(0)
    trainer.check()
    sizes_px = [h * w for h, w, _ in sizes]
    pix_f = list(torch.split(pix, sizes_px))
    tgt_f = list(torch.split(tgt, sizes_px))
    ref = _torch_pipeline_steps(start, specs, pix_f, tgt_f, cfg, steps, dev)
    for name, a, b, s0 in zip(("means", "tril", "opacity", "intensity"), params.tensors(), ref, start):
        assert rel(b, s0) > 0, name  # the reference loop moved it
        # the batch sums its frames' gradients in another order than the per-frame loop, and Adam
        # turns rounding-level gradients into full steps: the displacements agree to ~1e-5
        print(f"[train] {name}: displacement rel diff {rel(a - s0, b - s0):.3e}")
        assert rel(a - s0, b - s0) <= 1e-4, (name, rel(a - s0, b - s0))
    st = trainer.losses(0)
    assert torch.isfinite(st).all()


def test_trainer_graph_replay_equals_eager(cuda_device):
    from us3d_b200 import scenes
    from us3d_b200.train import TrainConfig, UltraGaussParameters, UltraGaussTrainer

    dev = cuda_device
    specs, pix = _specs(((96, 128, 0.25), (80, 80, 0.3)), seed=6)
    pix = pix.to(dev)
    sc = scenes.make_scene(15000, seed=6, cube_mm=32.0)
    tgt = torch.rand(pix.shape[0], generator=torch.Generator().manual_seed(1)).to(dev)
    out = []
    for graph in (False, True):
        params = UltraGaussParameters.from_points(sc.means.to(dev), sc.intensities.to(dev), init_scale_mm=0.8)
        tr = UltraGaussTrainer(params, [(specs, pix, tgt)], TrainConfig(lr=5e-3, ssim_weight=0.1), graph=graph)
        for _ in range(4):
            tr.step(0)
        tr.check()
        out.append([t.cpu().numpy() for t in params.tensors()])
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_refine_stats_kernel(cuda_device):
    from us3d_b200.refine import RefineStats

    dev = cuda_device
    g = torch.Generator().manual_seed(3)
    grads = torch.randn((5000, 3), generator=g)
    grads[::7] = 0.0
    st = RefineStats(5000, dev)
    for _ in range(3):
        st.accumulate(grads.to(dev))
    n = grads.norm(dim=1)
    assert torch.allclose(st.importance.cpu(), 3 * n, rtol=1e-6, atol=0)
    assert torch.equal(st.visits.cpu(), 3 * (n > 0).int())


def test_trainer_with_refinement(cuda_device):
    """Densification and pruning inside graph-replayed training: the Gaussian count changes,
    graphs are captured again, the capacity check holds, and training continues."""
    from us3d_b200 import scenes
    from us3d_b200.refine import RefineConfig
    from us3d_b200.train import TrainConfig, UltraGaussParameters, UltraGaussTrainer

    dev = cuda_device
    specs, pix = _specs(((96, 128, 0.25), (80, 80, 0.3)), seed=4)
    pix = pix.to(dev)
    sc = scenes.make_scene(20000, seed=4, cube_mm=32.0)
    params = UltraGaussParameters.from_points(sc.means.to(dev), sc.intensities.to(dev), init_scale_mm=0.8)
    tgt = torch.rand(pix.shape[0], generator=torch.Generator().manual_seed(9)).to(dev)
    rc = RefineConfig(every=2, start=2, stop=4, grad_threshold=1e-6, split_scale_mm=0.9, max_gaussians=24000)
    tr = UltraGaussTrainer(params, [(specs, pix, tgt)], TrainConfig(lr=1e-2), refine=rc)
    for _ in range(6):
        tr.step(0)
    tr.check()
    assert [r["step"] for r in tr.refine_log] == [2, 4]
    assert params.means.shape[0] == tr.refine_log[-1]["total"] != 20000
    assert all(r["cloned"] + r["split"] > 0 for r in tr.refine_log)
    assert params.means.shape[0] <= 24000
    for t in params.tensors():
        assert torch.isfinite(t).all()
    assert torch.isfinite(tr.losses(0)).all()


def test_trainer_checkpoint_resume_bit_identical(cuda_device, tmp_path):
    """A run saved after a refinement and resumed in a fresh trainer (from the initial
    parameters, so the loaded state has another number of Gaussians) takes the same steps bit
    for bit as the uninterrupted run: parameters, Adam moments, step count, refinement
    statistics and log, and the generators of the batch draws and of the refinement."""
    from us3d_b200 import scenes
    from us3d_b200.frames import DeviceFrameSource
    from us3d_b200.refine import RefineConfig
    from us3d_b200.train import TrainConfig, UltraGaussParameters, UltraGaussTrainer

    dev = cuda_device
    rng = np.random.default_rng(3)
    n, h, w = 6, 64, 80
    images = rng.integers(0, 255, (n, h, w), dtype=np.uint8)
    origin = np.stack([np.array([4.0 + 2.5 * k, 2.0, 16.0], np.float32) for k in range(n)])
    src = DeviceFrameSource(images, origin, np.array([0, 0, 1], np.float32), np.array([0, 1, 0], np.float32),
                            np.array([1, 0, 0], np.float32), 0.25, 0.25, device=dev)
    sc = scenes.make_scene(12000, seed=7, cube_mm=32.0)
    rc = RefineConfig(every=3, start=3, stop=9, grad_threshold=1e-7, split_scale_mm=0.9, max_gaussians=16000)

    def fresh():
        params = UltraGaussParameters.from_points(sc.means.to(dev), sc.intensities.to(dev), init_scale_mm=0.8)
        return params, UltraGaussTrainer.from_source(params, src, 3, TrainConfig(lr=1e-2), refine=rc, seed=5)

    pa, ta = fresh()
    for _ in range(10):
        ta.step(0)
    pb, tb = fresh()
    for _ in range(4):
        tb.step(0)
    tb.save(tmp_path / "ckpt.pt")
    assert [r["step"] for r in tb.refine_log] == [3]
    pc, tc = fresh()
    tc.load(tmp_path / "ckpt.pt")
    assert tc.steps_done == 4 and pc.means.shape[0] == pb.means.shape[0] != 12000
    for _ in range(6):
        tc.step(0)
    ta.check()
    tc.check()
    assert [r["step"] for r in tc.refine_log] == [r["step"] for r in ta.refine_log] == [3, 6, 9]
    assert tc.refine_log == ta.refine_log
    for x, y in zip(pa.tensors(), pc.tensors()):
        assert torch.equal(x, y)
    for x, y in zip(ta.optimizer.exp_avg + ta.optimizer.exp_avg_sq, tc.optimizer.exp_avg + tc.optimizer.exp_avg_sq):
        assert torch.equal(x, y)
