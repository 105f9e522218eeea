"""Synthetic workloads beyond the headline benchmark, run on one GPU and reported as JSON.

``python -m us3d_b200.workloads sweeps``    independent sweeps with their own Gaussian sets
                                            and frame sizes, batched into one launch sequence
                                            per step (captured as a CUDA graph) against the
                                            one-frame-per-launch form;
``python -m us3d_b200.workloads training``  end-to-end UltraGauss training with densification
                                            and pruning (layered point cloud, three crossing
                                            sweeps, targets rendered from a larger ground
                                            truth with Rayleigh speckle) against the
                                            one-frame-per-step form.

Every scene and sweep is seeded; the sizes of the full workloads are the defaults, and the
GPU tests run reduced versions of the same code.
"""

from __future__ import annotations

import argparse
import json
import math
import time
from dataclasses import dataclass
from typing import List, Optional

import torch

from . import scenes
from . import ultragauss as UG

CHI2, BETA, BG_A, BG_I = 7.815, 1e-4, 1e-6, 0.0


# ------------------------------------------------------------------------------------
# Independent sweeps with their own Gaussian sets
# ------------------------------------------------------------------------------------

@dataclass
class Sweep:
    first_gaussian: int
    n_gaussians: int
    size: int
    n_frames: int
    specs: List[UG.SliceSpec]


@dataclass
class SweepBatch:
    params: List[torch.Tensor]  # concatenated means, precision_tril, opacities, intensities
    sweeps: List[Sweep]
    specs: List[UG.SliceSpec]   # every frame, sweep by sweep, with its Gaussian set
    pixels: torch.Tensor        # (P,3) all frames
    d_image: torch.Tensor       # (P,) seeded upstream gradient


def make_sweep_batch(n_sweeps: int = 64, g_min: int = 10_000, g_max: int = 1_000_000, sizes=(128, 256, 384, 512),
                     frames_min: int = 8, frames_max: int = 64, fov_mm: float = 64.0, seed: int = 0,
                     device: Optional[torch.device] = None) -> SweepBatch:
    """Sweep s has G_s ~ log-uniform[g_min, g_max] Gaussians of the headline distributions
    (its own 64 mm cube scene, seed + 1 + s), a frame size drawn from ``sizes`` (square, pixel
    pitch fov_mm / size, so every frame covers the cube) and frames_min..frames_max frames of a
    linear sweep through its cube. Parameters are concatenated sweep by sweep; every frame
    names its sweep's Gaussian set."""
    g = torch.Generator().manual_seed(seed)
    u = torch.rand((n_sweeps,), generator=g, dtype=torch.float64)
    counts = torch.exp(math.log(g_min) + u * (math.log(g_max) - math.log(g_min))).round().long().tolist()
    size_idx = torch.randint(0, len(sizes), (n_sweeps,), generator=g).tolist()
    n_frames = torch.randint(frames_min, frames_max + 1, (n_sweeps,), generator=g).tolist()
    parts = [[], [], [], []]
    sweeps, specs, pix = [], [], []
    off = 0
    for s in range(n_sweeps):
        G = int(counts[s])
        sc = scenes.make_scene(G, seed=seed + 1 + s)
        for k, t in enumerate((sc.means, sc.precision_tril, sc.opacities, sc.intensities)):
            parts[k].append(t)
        size = int(sizes[size_idx[s]])
        F = int(n_frames[s])
        sw = scenes.linear_sweep(F, size, size, fov_mm / size, seed=seed + 1 + s, step_mm=min(2.0, 60.0 / F))
        ss = [UG.SliceSpec(f.height, f.width, f.lateral_spacing, f.axial_spacing, f.axial_near, f.lateral_col_offset,
                           f.origin, f.axis_lat, f.axis_ax, f.axis_ele, gaussian_set=(off, G)) for f in sw]
        sweeps.append(Sweep(off, G, size, F, ss))
        specs += ss
        pix += [f.pixels for f in sw]
        off += G
    dev = device or torch.device("cuda", torch.cuda.current_device())
    params = [torch.cat(p).to(dev).contiguous() for p in parts]
    pixels = torch.cat(pix).to(dev).contiguous()
    gd = torch.Generator().manual_seed(seed + 99)
    d_image = (torch.randn(pixels.shape[0], generator=gd) / 1e6).to(dev)
    return SweepBatch(params, sweeps, specs, pixels, d_image)


def run_sweeps(batch: SweepBatch, steps: int = 3, warmup: int = 2, plain_steps: int = 1) -> dict:
    """Times the batched step (one slice-culled binning, forward and adjoint launch sequence
    over every frame of every sweep, replayed from a CUDA graph) and the plain form (one
    frame per launch sequence with its own sweep's parameters, the reference's calling
    pattern), both with CUDA events; returns frames/s of each."""
    from .batch import GraphedTrainingStep

    dev = batch.pixels.device
    n_frames = len(batch.specs)
    zeros = torch.zeros_like(batch.d_image)
    step = GraphedTrainingStep(batch.specs, dev, batch.params, batch.pixels,
                               lambda img, alpha, depth: (batch.d_image, zeros, zeros))
    for _ in range(warmup):
        step.replay()
    torch.cuda.synchronize(dev)
    st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st.record()
    for _ in range(steps):
        step.replay()
    en.record()
    en.synchronize()
    ms = st.elapsed_time(en) / steps
    total = step.check()
    step_result = dict(ms_per_step=round(ms, 3), frames_per_s=round(n_frames / (ms / 1e3), 1),
                       instances=int(total))
    del step
    torch.cuda.empty_cache()

    # plain: one frame at a time with its sweep's own parameter slices
    means, tril, opac, inten = batch.params
    tables, pix_off = [], 0
    for sw in batch.sweeps:
        a, b = sw.first_gaussian, sw.first_gaussian + sw.n_gaussians
        for sp in sw.specs:
            single = UG.SliceSpec(sp.height, sp.width, sp.lateral_spacing, sp.axial_spacing, sp.axial_near,
                                  sp.lateral_col_offset, sp.origin, sp.axis_lat, sp.axis_ax, sp.axis_ele)
            P = sp.height * sp.width
            tables.append((UG.build_frame_table([single], dev), a, b, pix_off, P))
            pix_off += P

    def plain_pass():
        for ft, a, b, po, P in tables:
            bb = UG.bin_gaussians(means[a:b], tril[a:b], opac[a:b], inten[a:b], ft, CHI2, BETA, True)
            px = batch.pixels[po:po + P]
            img, alpha, depth, _ = UG.forward(bb, px, BG_A, BG_I)
            z = torch.zeros_like(img)
            UG.backward(bb, px, batch.d_image[po:po + P], z, z, alpha, BG_A, BG_I)

    plain_pass()
    torch.cuda.synchronize(dev)
    st.record()
    for _ in range(plain_steps):
        plain_pass()
    en.record()
    en.synchronize()
    ms_plain = st.elapsed_time(en) / plain_steps
    return dict(workload=f"{len(batch.sweeps)} independent sweeps, own Gaussian sets "
                         f"({min(s.n_gaussians for s in batch.sweeps)}..{max(s.n_gaussians for s in batch.sweeps)} "
                         f"Gaussians), frame sizes {sorted({s.size for s in batch.sweeps})}, {n_frames} frames",
                gaussians=int(means.shape[0]), frames=n_frames, pixels=int(batch.pixels.shape[0]),
                batched=step_result,
                plain=dict(ms_per_pass=round(ms_plain, 3), frames_per_s=round(n_frames / (ms_plain / 1e3), 1)),
                batched_over_plain=round(ms_plain / ms, 3))


# ------------------------------------------------------------------------------------
# End-to-end training with densification and pruning
# ------------------------------------------------------------------------------------

def layered_point_cloud(n: int, seed: int = 0, extent_mm=(64.0, 64.0, 64.0), n_layers: int = 8,
                        n_inclusions: int = 40, radius_mm=(2.0, 8.0)):
    """Tissue-like point cloud: n points, half of them in n_layers horizontal layers
    (depth bands of random thickness 2-6 mm, each with its own echogenicity), half in
    n_inclusions spheres of radius U(radius_mm) (bright or dark), uniform inside; every point
    carries an intensity in [0, 1] (its structure's echogenicity plus 5 % noise)."""
    g = torch.Generator().manual_seed(seed)
    ext = torch.tensor(extent_mm)
    n_layer = n // 2
    n_inc = n - n_layer
    tops = torch.sort(torch.rand((n_layers,), generator=g) * ext[1] * 0.85).values
    thick = 2.0 + 4.0 * torch.rand((n_layers,), generator=g)
    layer_int = 0.2 + 0.6 * torch.rand((n_layers,), generator=g)
    which = torch.randint(0, n_layers, (n_layer,), generator=g)
    p_layer = torch.rand((n_layer, 3), generator=g) * ext
    p_layer[:, 1] = tops[which] + thick[which] * torch.rand((n_layer,), generator=g)
    i_layer = layer_int[which]
    centres = (0.1 + 0.8 * torch.rand((n_inclusions, 3), generator=g)) * ext
    radii = radius_mm[0] + (radius_mm[1] - radius_mm[0]) * torch.rand((n_inclusions,), generator=g)
    inc_int = torch.where(torch.rand((n_inclusions,), generator=g) < 0.5, torch.tensor(0.9), torch.tensor(0.05))
    wi = torch.randint(0, n_inclusions, (n_inc,), generator=g)
    d = torch.randn((n_inc, 3), generator=g)
    d = d / d.norm(dim=1, keepdim=True).clamp_min(1e-12)
    r = torch.rand((n_inc,), generator=g).pow(1.0 / 3.0) * radii[wi]
    p_inc = centres[wi] + d * r[:, None]
    pts = torch.cat([p_layer, p_inc])
    inten = torch.cat([i_layer, inc_int[wi]])
    inten = (inten + 0.05 * torch.randn((n,), generator=g)).clamp(0.0, 1.0)
    pts = torch.minimum(torch.maximum(pts, torch.zeros(3)), ext)
    return pts.contiguous(), inten.contiguous()


def crossing_sweeps(n_frames: int, size: int, spacing_mm: float, seed: int = 0, cube_mm: float = 64.0):
    """Three sweeps through the cube along crossing directions (elevation along z, x and the
    xz diagonal), n_frames in total, each frame tilted N(0, 2 deg) and centred in the cube."""
    g = torch.Generator().manual_seed(seed + 7)
    per = [n_frames // 3 + (1 if k < n_frames % 3 else 0) for k in range(3)]
    out = []
    c = torch.tensor([cube_mm / 2] * 3)
    eles = [torch.tensor([0.0, 0.0, 1.0]), torch.tensor([1.0, 0.0, 0.0]),
            torch.tensor([1.0, 0.0, 1.0]) / math.sqrt(2.0)]
    ax0 = torch.tensor([0.0, 1.0, 0.0])
    depth = size * spacing_mm
    for k, n in enumerate(per):
        ele0 = eles[k]
        lat0 = torch.linalg.cross(ax0, ele0)
        lat0 = lat0 / lat0.norm()
        for f in range(n):
            t = (f + 0.5) / max(n, 1) - 0.5
            tilt = float(torch.randn((), generator=g)) * math.radians(2.0)
            R = scenes._rot_about(lat0, tilt)
            ax = R @ ax0
            ele = R @ ele0
            centre = c + ele0 * (t * cube_mm * 0.9)
            origin = centre - ax * (depth * 0.5)
            pix = scenes.slice_pixels(origin, lat0, ax, size, size, spacing_mm, spacing_mm, 0.0, (size - 1) * 0.5)
            out.append(scenes.Slice(size, size, spacing_mm, spacing_mm, 0.0, (size - 1) * 0.5, origin, lat0.clone(),
                                    ax, ele, pix))
    return out


def speckle_targets(gt: scenes.GaussianScene, frames, device, seed: int = 0, sigma: float = 0.3,
                    chunk: int = 16) -> torch.Tensor:
    """Targets: the ground truth rendered (batched forward) times Rayleigh speckle of scale
    sigma (normalised to unit mean), clipped to [0, 1]; (n_frames, H*W) on the device."""
    g = torch.Generator(device=device)
    g.manual_seed(seed + 11)
    out = []
    params = [gt.means.to(device), gt.precision_tril.to(device).contiguous(), gt.opacities.to(device),
              gt.intensities.to(device)]
    mean_rayleigh = sigma * math.sqrt(math.pi / 2.0)
    for s in range(0, len(frames), chunk):
        fr = frames[s:s + chunk]
        specs = [UG.SliceSpec(f.height, f.width, f.lateral_spacing, f.axial_spacing, f.axial_near,
                              f.lateral_col_offset, f.origin, f.axis_lat, f.axis_ax, f.axis_ele) for f in fr]
        ft = UG.build_frame_table(specs, device)
        pix = torch.cat([f.pixels for f in fr]).to(device)
        b = UG.bin_gaussians(*params, ft, CHI2, BETA, True, slice_cull_pixels=pix)
        img, _, _, _ = UG.forward(b, pix, BG_A, BG_I, want_counts=False)
        u = torch.rand(img.shape, generator=g, device=device).clamp_min(1e-12)
        ray = sigma * torch.sqrt(-2.0 * torch.log(u)) / mean_rayleigh
        out.append((img * ray).clamp(0.0, 1.0).reshape(len(fr), -1))
    return torch.cat(out)


def _train_curve(make_trainer, params, steps: int, batch: int, evals: int, l1_on_held) -> dict:
    """Trains ``steps`` steps, pausing ``evals`` times to take the held-out L1 (outside the
    timed region); returns frames/s over the training time alone, the curve of (seconds,
    frames, held-out L1) and the trainer's refinement log."""
    trainer = make_trainer(params)
    dev = params.means.device
    curve = [(0.0, 0, round(l1_on_held(params), 6))]
    every = max(1, steps // max(1, evals))
    st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms, done = 0.0, 0
    while done < steps:
        n = min(every, steps - done)
        torch.cuda.synchronize(dev)
        st.record()
        for _ in range(n):
            trainer.step(0)
        en.record()
        en.synchronize()
        ms += st.elapsed_time(en)
        done += n
        curve.append((round(ms / 1e3, 3), done * batch, round(l1_on_held(params), 6)))
    trainer.check()
    out = dict(steps=steps, frames=steps * batch, seconds=round(ms / 1e3, 3),
               frames_per_s=round(steps * batch / (ms / 1e3), 1), held_out_l1=curve[-1][2], curve=curve,
               gaussians_final=int(params.means.shape[0]), refinements=list(getattr(trainer, "refine_log", [])))
    del trainer
    torch.cuda.empty_cache()
    return out


def _seconds_to(curve, target: float) -> Optional[float]:
    """First time (linear between evaluations) at which the held-out L1 reaches target."""
    for (t0, _, l0), (t1, _, l1) in zip(curve, curve[1:]):
        if l1 <= target:
            return round(t0 + (t1 - t0) * ((l0 - target) / (l0 - l1) if l0 > l1 else 1.0), 3)
    return None


def run_training(n_init: int = 2_000_000, n_gt: int = 4_000_000, n_frames: int = 1500, size: int = 512,
                 spacing_mm: float = 0.15, batch: int = 16, steps: int = 5000, refine_every: int = 500,
                 plain_frames: int = 16000, seed: int = 0, max_gaussians: int = 3_000_000,
                 densify_fraction: float = 0.01, evals: int = 20, device: Optional[torch.device] = None) -> dict:
    """The end-to-end training workload: initial Gaussians from the layered point cloud
    (n_init points), targets from an n_gt-Gaussian ground truth of the same structures with
    Rayleigh speckle, n_frames frames of size^2 px at spacing_mm from three crossing sweeps,
    batches of ``batch`` frames per step drawn on the device, forward + loss + backward +
    Adam per step (graph-replayed), densify (the top ``densify_fraction`` by importance) and
    prune every ``refine_every`` steps during the first 60 % of the steps. Three runs from the same initial state: the batched
    form at the reference's learning rate (1e-3), the batched form at sqrt(batch) times it
    (Adam's step does not grow with the batch, so a 16-frame step otherwise moves as far as a
    1-frame step), and the one-frame-per-step form (the reference's pattern) for
    ``plain_frames`` frames. Reports frames/s, the step's HBM rate from its algorithmic bytes,
    held-out L1 curves on 64 frames, and the training time each batched run needs to reach the
    plain form's final held-out L1 (matched accuracy)."""
    from .frames import DeviceFrameSource
    from .refine import RefineConfig
    from .train import TrainConfig, UltraGaussParameters, UltraGaussTrainer

    dev = device or torch.device("cuda", torch.cuda.current_device())
    t0 = time.perf_counter()
    gt_pts, gt_int = layered_point_cloud(n_gt, seed=seed + 1)
    gt = scenes.make_scene(n_gt, seed=seed + 2, log_scale_mean=math.log(0.35), log_scale_std=0.3)
    gt.means, gt.intensities = gt_pts, gt_int
    frames = crossing_sweeps(n_frames, size, spacing_mm, seed=seed)
    targets = speckle_targets(gt, frames, dev, seed=seed)
    del gt
    source = DeviceFrameSource((targets * 255.0).round().to(torch.uint8).reshape(n_frames, size, size),
                               torch.stack([f.origin for f in frames]), torch.stack([f.axis_lat for f in frames]),
                               torch.stack([f.axis_ax for f in frames]), torch.stack([f.axis_ele for f in frames]),
                               spacing_mm, spacing_mm, device=dev)
    del targets
    torch.cuda.empty_cache()
    prep_s = time.perf_counter() - t0
    init_pts, init_int = layered_point_cloud(n_init, seed=seed + 3)

    def fresh():
        return UltraGaussParameters.from_points(init_pts.to(dev), init_int.to(dev), init_scale_mm=0.5,
                                                init_opacity=0.1)

    held = torch.arange(0, n_frames, max(1, n_frames // 64), device=dev)[:64]

    def l1_on_held(p):
        tab, pix, tgt = source.batch(held)
        b = UG.bin_gaussians(p.means, p.raw_precision_tril, p.raw_opacities.reshape(-1),
                             p.raw_intensities.reshape(-1), tab, CHI2, BETA, True, slice_cull_pixels=pix,
                             logit_attributes=True)
        img, _, _, _ = UG.forward(b, pix, BG_A, BG_I, want_counts=False)
        return float((img - tgt).abs().mean())

    # refinement during the first 60 % of the steps, as the schedule it follows (every 2500 of
    # 30k iterations, from 1k to 20k): the rest of the run settles the refined set
    rcfg = RefineConfig(every=refine_every, start=refine_every, stop=int(steps * 0.6), max_gaussians=max_gaussians,
                        densify_fraction=densify_fraction)
    runs = {}
    for name, lr in (("batched", 1.0e-3), ("batched_lr_sqrt_batch", 1.0e-3 * math.sqrt(batch))):
        runs[name] = _train_curve(
            lambda p, lr=lr: UltraGaussTrainer.from_source(p, source, batch, TrainConfig(lr=lr), refine=rcfg,
                                                            seed=seed), fresh(), steps, batch, evals, l1_on_held)
        runs[name]["lr"] = lr
    # algorithmic HBM bytes of a step at the final size: parameters read by binning, forward and
    # backward, gradients written, Adam's 28 bytes per parameter element, pixels and targets
    P = size * size
    for r in runs.values():
        G = r["gaussians_final"]
        bytes_step = G * 44 * 3 + G * 44 + G * 11 * 28 + batch * P * (12 + 1 + 12 + 12)
        r["hbm_gbs_algorithmic"] = round(bytes_step * r["steps"] / r["seconds"] / 1e9, 1)
    plain = _train_curve(lambda p: UltraGaussTrainer.from_source(p, source, 1, TrainConfig(), seed=seed + 1), fresh(),
                         int(plain_frames), 1, evals, l1_on_held)
    plain["lr"] = 1.0e-3
    target = plain["held_out_l1"]
    matched = {name: dict(seconds_to_plain_final_l1=_seconds_to(r["curve"], target),
                          plain_seconds=plain["seconds"]) for name, r in runs.items()}
    return dict(workload=f"UltraGauss training: {n_init} initial Gaussians (layered point cloud + inclusions), "
                         f"{n_frames} frames {size}^2 px @ {spacing_mm} mm from three crossing sweeps, targets from "
                         f"{n_gt} ground-truth Gaussians with Rayleigh speckle, {batch} frames/step, "
                         f"densify (top {densify_fraction:.0%}) / prune every {refine_every} steps",
                preparation_s=round(prep_s, 2), held_out_l1_at_start=runs["batched"]["curve"][0][2], **runs,
                plain=plain, matched_accuracy=dict(target_held_out_l1=target, **matched),
                batched_over_plain_frames_per_s=round(runs["batched"]["frames_per_s"] / plain["frames_per_s"], 3))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=["sweeps", "training"])
    ap.add_argument("--scale", type=float, default=1.0, help="fraction of the full workload's sizes")
    ap.add_argument("--steps", type=int, default=None)
    a = ap.parse_args()
    torch.cuda.set_device(0)
    if a.workload == "sweeps":
        n = max(2, int(round(64 * a.scale)))
        b = make_sweep_batch(n_sweeps=n, g_max=int(max(20_000, 1_000_000 * min(1.0, a.scale * 2))))
        out = run_sweeps(b, steps=a.steps or 3)
    else:
        s = a.scale
        out = run_training(n_init=int(2_000_000 * s), n_gt=int(4_000_000 * s), n_frames=max(48, int(1500 * s)),
                           steps=a.steps or int(5000 * s), refine_every=max(10, int(500 * s)),
                           plain_frames=int(16000 * s), max_gaussians=int(3_000_000 * s))
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
