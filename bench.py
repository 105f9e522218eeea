"""Benchmark: UltraGauss slice splatting fwd+bwd frames/s on B200 (batched vs plain).

Workload (headline scene): 1,000,000 anisotropic Gaussians in a 64 mm cube (means uniform,
log-scales N(log 1 mm, 0.3), random unit quaternions, intensity U(0,1), opacity
sigmoid(N(0,1)), seed 0); frames 512x512 px at 0.125 mm from a linear sweep (2 mm steps,
tilt N(0, 2 deg)); 16 frames per step; L1 loss against seeded U(0,1) targets. A step is
fwd + loss gradient + bwd of all 16 frames (gradients summed over frames).

  value      batched form: one binning, one forward and one adjoint launch sequence for the
             16 frames, inputs resident in HBM;
  plain      one frame per launch sequence (the reference's calling pattern);
  e2e        batched form through the public autograd API with pinned host inputs: per step
             H2D of parameters, pixel positions and targets, D2H of loss and gradients.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
Multi-GPU (replicas over frames, no collective): torchrun --nproc-per-node N bench.py --gpus N
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "ultrasound-3d-reconstruction_b200"))
sys.path.insert(0, str(ROOT))

METRIC = "fwd+bwd frames/s @1M Gaussians 512² (batched vs plain, 1 B200); % HBM roofline"
UNIT = "frames/s"
BP, BG, BO, BD = 44, 44, 12, 12  # algorithmic bytes per Gaussian / pixel (params, grads, outputs, upstream)

# Per-frame ncu figures of each stage's kernels, from one capture of a 4-frame launch of the
# same scene (ncu --set full; profiles/ultragauss_*_4frames.md), keyed by stage and by that
# stage's kernel variant (0 one pixel per FP32 instruction, 1 packed FP32x2 pairs):
#   traffic: dram__bytes_read.sum + dram__bytes_write.sum per frame (the backward stage is the
#            shading adjoint + the per-Gaussian reduce_kernel), scaled to the launch's frames;
#   inst:    (smsp__inst_executed.sum per frame, per launch) -- the reduction runs once per launch;
#   fma:     sm__pipe_fma_cycles_active share of the shading kernel.
# A variant without a capture has no entry and reports no issue figure.
NCU_STAGE = {
    "ug_forward": {
        0: dict(traffic=(52.290304e6 + 4.972288e6) / 4, inst=(466223281 / 4, 0.0), fma=0.5092),
        1: dict(traffic=(52.252416e6 + 4.260352e6) / 4, inst=(487111780 / 4, 0.0), fma=0.5661),
    },
    "ug_backward": {
        0: dict(traffic=(100.252416e6 + 114.988544e6 + 156.020480e6 + 28.401920e6) / 4,
                inst=(594881545 / 4, 21e6), fma=0.6857),
        1: dict(traffic=(99.148032e6 + 114.697984e6 + 156.020480e6 + 28.401920e6) / 4,
                inst=(377437123 / 4, 21e6), fma=0.7181),
    },
}
SM_COUNT, SCHEDULERS_PER_SM = 148, 4


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--gaussians", type=int, default=1_000_000)
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--spacing", type=float, default=0.125)
    ap.add_argument("--frames-per-step", type=int, default=16)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-train", action="store_true", help="skip the training-step measurement")
    ap.add_argument("--launch-shape", default=None,
                    help="forward batch / backward threads [/ backward variant [/ forward variant]] (0 scalar, 1 packed), e.g. "
                         "512/256/1, instead of autotuning")
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload_config(a, world):
    return {
        "workload": (f"ultragauss slice splatting fwd+bwd, {a.gaussians} Gaussians (64 mm cube), "
                     f"{a.size}x{a.size} px @ {a.spacing} mm, {a.frames_per_step} frames/step per GPU"),
        "gaussians": a.gaussians,
        "frame_px": [a.size, a.size],
        "pixel_mm": a.spacing,
        "frames_per_step": a.frames_per_step * world,
        "parallelism": f"replicas{world}",
        "l2": "inputs larger than L2 (params 44 MB + pixel positions 50 MB + per-step instance lists)",
    }


class Clocks:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        # the timed region starts once the sampler is running (first sample written)
        t0 = time.time()
        while self.proc is not None and self.proc.poll() is None and time.time() - t0 < 5.0:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.01)
        self.skip = 1 if self.proc is not None and os.path.getsize(self.path) > 0 else 0
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        # the first sample precedes the timed region
        for line in open(self.path).readlines()[getattr(self, "skip", 0):]:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def build_inputs(a, device, rank):
    import torch

    from us3d_b200 import scenes
    from us3d_b200 import ultragauss as UG

    sc = scenes.make_scene(a.gaussians, seed=0)
    n_pool = max(2 * a.frames_per_step, 32)
    sweep = scenes.linear_sweep(n_pool, a.size, a.size, a.spacing, seed=rank, step_mm=64.0 / n_pool)
    specs = [UG.SliceSpec(f.height, f.width, f.lateral_spacing, f.axial_spacing, f.axial_near, f.lateral_col_offset,
                          f.origin, f.axis_lat, f.axis_ax, f.axis_ele) for f in sweep]
    pixels = torch.cat([f.pixels for f in sweep]).to(device)
    g = torch.Generator().manual_seed(1234 + rank)
    targets = torch.rand((n_pool * a.size * a.size,), generator=g).to(device)
    params = [sc.means.to(device), sc.precision_tril.to(device).contiguous(), sc.opacities.to(device),
              sc.intensities.to(device)]
    return sc, specs, pixels, targets, params, n_pool


def run_b200(a):
    import torch
    import torch.distributed as dist

    from us3d_b200 import _lib
    from us3d_b200 import ultragauss as UG
    from us3d_b200.dist import max_over_ranks

    rank, world, local = dist_env()
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    L = _lib.load()
    sc, specs, pixels, targets, params, n_pool = build_inputs(a, dev, rank)
    F = a.frames_per_step
    P1 = a.size * a.size
    batches = []
    for s in range(0, n_pool, F):
        ft = UG.build_frame_table(specs[s:s + F], dev)
        batches.append((ft, pixels[s * P1:(s + F) * P1], targets[s * P1:(s + F) * P1]))
    single_tables = [UG.build_frame_table([sp], dev) for sp in specs]
    grad_bufs = [torch.empty_like(p) for p in params]
    scratch = [None]
    inst_per_frame = []

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def l1_grad(img, tgt):
        return torch.sign(img - tgt) / img.numel()

    def batched_step(i):
        ft, pix, tgt = batches[i % len(batches)]
        b = UG.bin_gaussians(*params, ft, 7.815, 1e-4, True, slice_cull_pixels=pix)
        img, alpha, depth, _ = UG.forward(b, pix, 1e-6, 0.0, want_counts=False)
        dI = l1_grad(img, tgt)
        z = torch.zeros_like(img)
        UG.backward(b, pix, dI, z, z, alpha, 1e-6, 0.0, out=grad_bufs)
        return b

    def plain_step(i):
        acc = None
        for f in range(F):
            k = (i * F + f) % n_pool
            pix = pixels[k * P1:(k + 1) * P1]
            tgt = targets[k * P1:(k + 1) * P1]
            b = UG.bin_gaussians(*params, single_tables[k], 7.815, 1e-4, True)
            img, alpha, depth, counts = UG.forward(b, pix, 1e-6, 0.0)
            dI = l1_grad(img, tgt)
            z = torch.zeros_like(img)
            g = UG.backward(b, pix, dI, z, z, alpha, 1e-6, 0.0)
            if acc is None:
                acc = [x.clone() for x in g]
            else:
                for x, y in zip(acc, g):
                    x.add_(y)
        return acc

    def timed(fn, steps, warm):
        for i in range(warm):
            fn(i)
        barrier()
        st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        st.record()
        for i in range(steps):
            fn(warm + i)
        en.record()
        barrier()
        return max_over_ranks(st.elapsed_time(en), device=dev)

    # -- launch-shape autotuning on the first batch (untimed; changes no result) --
    from us3d_b200.batch import autotune_launch, set_backward_variant, set_forward_variant, set_launch_config

    if a.launch_shape:
        launch_shape = tuple(int(x) for x in a.launch_shape.split("/"))
        launch_shape = (*launch_shape, 1, 0)[:4] if len(launch_shape) == 2 else \
            ((*launch_shape, 0) if len(launch_shape) == 3 else launch_shape)
        set_launch_config(launch_shape[0], launch_shape[1])
        set_backward_variant(launch_shape[2])
        set_forward_variant(launch_shape[3])
        tuned = {}
    else:
        tuned = autotune_launch(batches[0][0], params, batches[0][1])
        launch_shape = min(tuned, key=tuned.get)

    # -- warm-up + stage selection for the roofline (untimed) --
    stage_ms = {}
    for stage in ("ug_bin", "ug_forward", "ug_backward"):
        _lib.check(L.us3d_profile_stage(stage.encode(), 8), "profile")
        b = batched_step(0)
        n = __import__("ctypes").c_int32(0)
        tot = __import__("ctypes").c_double(0)
        _lib.check(L.us3d_profile_collect(__import__("ctypes").byref(n), __import__("ctypes").byref(tot)), "collect")
        stage_ms[stage] = tot.value / max(n.value, 1)
        inst_per_frame.append(b.total / F)
    dominant = max(stage_ms, key=stage_ms.get)
    _lib.check(L.us3d_profile_stage(dominant.encode(), a.steps + 4), "profile")

    launches0 = L.us3d_launch_count()
    with Clocks(local) as clk:
        ms_batched = timed(batched_step, a.steps, a.warmup)
    launches = L.us3d_launch_count() - launches0
    import ctypes

    n = ctypes.c_int32(0)
    tot = ctypes.c_double(0)
    _lib.check(L.us3d_profile_collect(ctypes.byref(n), ctypes.byref(tot)), "collect")
    _lib.check(L.us3d_profile_stage(None, 0), "profile off")
    # launches counted include the warm-up steps; keep only the timed ones
    per_step_launches = launches / (a.steps + a.warmup)
    gpu_launches = int(round(per_step_launches * a.steps))
    stage_avg_ms = tot.value / max(n.value, 1)
    clocks = clk.summary()

    # The same batched step captured once per frame batch as a CUDA graph and replayed (no
    # host round trip or launch gaps inside a step); the overflow flags are checked after.
    from us3d_b200.batch import GraphedTrainingStep

    graphed = []
    for ft_k, (ft, pix, tgt) in enumerate(batches):
        graphed.append(GraphedTrainingStep(specs[ft_k * F:(ft_k + 1) * F], dev, params, pix,
                                           lambda img, alpha, depth, tgt=tgt: (l1_grad(img, tgt), torch.zeros_like(img),
                                                                               torch.zeros_like(img)),
                                           grads=grad_bufs))

    def graphed_step(i):
        graphed[i % len(graphed)].replay()

    with Clocks(local) as clk_g:
        ms_graphed = timed(graphed_step, a.steps, a.warmup)
    for gs in graphed:
        gs.check()
    uncaptured_value = a.steps * F * world / (ms_batched / 1e3)
    if ms_graphed < ms_batched:
        ms_batched = ms_graphed
        clocks = clk_g.summary()

    frames_total = a.steps * F * world
    value = frames_total / (ms_batched / 1e3)
    I = statistics.mean(inst_per_frame)
    G = a.gaussians
    P = P1
    alg = {
        "ug_backward": G * (BP + BG) + I * 5 + P * (BO + BD),
        "ug_forward": I * 5 + P * BO,
        "ug_bin": G * BP + I * 13,
    }[dominant] * F
    peaks = json.load(open(ROOT / "MEASURED_PEAKS.json")) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = alg / (stage_avg_ms / 1e3) / 1e9
    variants = {"ug_forward": launch_shape[3], "ug_backward": launch_shape[2]}
    traffic = NCU_STAGE.get(dominant, {}).get(variants.get(dominant), {}).get("traffic")
    roofline = {"bound": "hbm", "kernel": dominant, "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": int(traffic * F) if traffic else None,
                "traffic_source": "ncu dram bytes of a 4-frame launch scaled to the launch's frames" if traffic else None,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks else "fallback 6650 GB/s",
                "stage_ms": {k: round(v, 4) for k, v in stage_ms.items()},
                "algorithmic_bytes_per_launch": int(alg)}
    # The whole step against the same peak, with the per-frame algorithmic bytes of the forward
    # (params once, instance key + value written and read, outputs) plus the backward (params
    # and gradients, instance list, saved outputs and upstream gradients).
    b_frame = (G * BP + I * 16 + P * BO) + (G * (BP + BG) + I * 4 + P * (BO + BD))
    step_gbs = b_frame * frames_total / (ms_batched / 1e3) / 1e9
    roofline["step"] = {"bytes_per_frame": int(b_frame), "achieved": round(step_gbs, 2),
                        "frac": round(step_gbs / peak, 4)}
    roofline["issue"] = issue_roofline(stage_ms, F, clocks, variants)

    out = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": round(ms_batched / a.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded headline scene (no dataset offline); targets U(0,1)",
        "config": workload_config(a, world), "instances_per_frame": round(I, 1), "roofline": roofline,
        "clocks": clocks, "gpu_launches": gpu_launches,
        "batched_form": "CUDA-graph replay of bin + forward + L1 gradient + backward per 16-frame batch",
        "launch_config": {"forward_batch": launch_shape[0], "backward_threads": launch_shape[1],
                          "backward_variant": ["scalar fp32", "packed fp32x2"][launch_shape[2]],
                          "forward_variant": ["scalar fp32", "packed fp32x2"][launch_shape[3]],
                          "autotune_ms_per_step": {"/".join(map(str, k)): round(v, 3) for k, v in tuned.items()}},
        "uncaptured": {"value": round(uncaptured_value, 3), "unit": UNIT,
                       "note": "same step launched from Python with one instance-total readback; "
                               "the roofline stage times come from this run's CUDA events"},
    }

    if not a.no_train:
        out["train_step"] = measure_train_step(a, params, specs, batches, F, world, timed)

    if not a.no_plain:
        steps_p = max(2, a.steps // 2)
        ms_plain = timed(plain_step, steps_p, 1)
        plain_value = steps_p * F * world / (ms_plain / 1e3)
        out["plain"] = {"value": round(plain_value, 3), "unit": UNIT, "ms_per_frame": round(ms_plain / (steps_p * F), 4)}
        out["batched_over_plain"] = round(value / plain_value, 3)

    if not a.no_e2e:
        out["e2e"] = run_e2e(a, dev, sc, specs, n_pool, world, rank, barrier)

    if rank == 0 and world == 1 and not a.no_cpu:
        out["cpu_baseline"] = cpu_baseline(a, sc, specs)
        out["cpu_baseline_dense_fallback"] = cpu_baseline_dense()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def issue_roofline(stage_ms, frames_per_launch, clocks, variants):
    """The bound the shading kernels actually meet: warp instructions issued per second
    against the GPU's issue ceiling (148 SMs x 4 schedulers x 1 warp instruction per clock at
    the median SM clock sampled during the timed region), per stage, from the instruction
    counts of the committed ncu capture of the stage's kernel variant scaled to the launch's
    frames and this run's CUDA-event stage times."""
    mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
    ceiling = SM_COUNT * SCHEDULERS_PER_SM * mhz * 1e6  # warp instructions / s
    out = {"bound": "instruction issue", "unit": "warp inst/s", "sm_mhz": mhz, "peak": ceiling,
           "source": "smsp__inst_executed.sum per frame of a 4-frame ncu capture (profiles/) x frames per launch "
                     "/ CUDA-event stage time; peak = 148 SMs x 4 schedulers x median SM clock"}
    for stage, by_variant in NCU_STAGE.items():
        ms = stage_ms.get(stage)
        fig = by_variant.get(variants.get(stage))
        if not ms or fig is None:
            continue
        per_frame, per_launch = fig["inst"]
        inst = per_frame * frames_per_launch + per_launch
        achieved = inst / (ms / 1e3)
        out[stage] = {"achieved": round(achieved, 1), "frac": round(achieved / ceiling, 4),
                      "warp_inst_per_launch": int(inst), "stage_ms": round(ms, 4), "variant": variants.get(stage),
                      "fma_pipe_busy": fig["fma"]}
    return out


def measure_train_step(a, params, specs, batches, F, world, timed):
    """The whole training step of the reference's loop (activations, L1 loss, backward, Adam
    over all parameters) on the bench's batches: forward + loss + backward replayed from a CUDA
    graph per batch, Adam one launch; the parameters are raw (logit) copies of the scene's."""
    import torch

    from us3d_b200.train import TrainConfig, UltraGaussParameters, UltraGaussTrainer

    tp = UltraGaussParameters(params[0].clone(), params[1].clone(), torch.logit(params[2].clamp(1e-6, 1 - 1e-6)),
                              torch.logit(params[3].clamp(1e-6, 1 - 1e-6)))
    trainer = UltraGaussTrainer(tp, [(specs[k * F:(k + 1) * F], pix, tgt) for k, (ft, pix, tgt) in enumerate(batches)],
                                TrainConfig())

    def train_step(i):
        trainer.step(i % len(batches))

    # every batch's graph is captured during the warm-up (its first step)
    ms_train = timed(train_step, a.steps, max(a.warmup, len(batches)))
    trainer.check()
    result = {"value": round(a.steps * F * world / (ms_train / 1e3), 3), "unit": UNIT,
              "ms_per_step": round(ms_train / a.steps, 4),
              "step": "bin (logistic activation fused) + forward + per-frame L1 loss + backward with the fused loss "
                      "gradient (CUDA-graph replay) + Adam over all 4 parameter tensors (one launch)"}
    del trainer, tp
    torch.cuda.synchronize()
    return result


def run_e2e(a, dev, sc, specs, n_pool, world, rank, timed_barrier):
    """End to end through the public autograd API: every step copies its inputs (Gaussian
    parameters, pixel positions, targets) from pinned host memory and reads its loss and
    gradients back. The next step's inputs are copied on a second stream while the current
    step computes (double buffering), and a step's loss and gradients go back to the host on a
    third stream while the next step computes; the timed region ends after the last of those
    copies. After a synchronised priming pass the renderers run without a per-step
    instance-total readback, and their overflow flags are checked after the timed region."""
    import torch

    from us3d_b200 import scenes
    from us3d_b200 import ultragauss as UG
    from us3d_b200.batch import UltraGaussBatchRenderer
    from us3d_b200.dist import max_over_ranks

    F = a.frames_per_step
    P1 = a.size * a.size
    host = [sc.means.pin_memory(), sc.precision_tril.contiguous().pin_memory(), sc.opacities.pin_memory(),
            sc.intensities.pin_memory()]
    sweep_pix = torch.cat([scenes.slice_pixels(s.origin, s.axis_lat, s.axis_ax, s.height, s.width, s.lateral_spacing,
                                               s.axial_spacing, s.axial_near, s.lateral_col_offset)
                           for s in specs]).pin_memory()
    g = torch.Generator().manual_seed(99 + rank)
    tgt_host = torch.rand((n_pool * P1,), generator=g).pin_memory()
    renderers = [UltraGaussBatchRenderer(specs[s:s + F], dev) for s in range(0, n_pool, F)]
    copy_stream = torch.cuda.Stream(device=dev)
    d2h_stream = torch.cuda.Stream(device=dev)
    compute = torch.cuda.current_stream()
    # two slots of device input buffers (refilled in place) and of pinned result buffers; a
    # step waits on the host until the results of the step two before it have arrived, as a
    # loop that reads every loss does, which also bounds how far the host runs ahead
    slots = [dict(step=-1, ready=torch.cuda.Event(), free=torch.cuda.Event(), landed=torch.cuda.Event(),
                  ps=[torch.empty(x.shape, dtype=x.dtype, device=dev) for x in host],
                  pix=torch.empty((F * P1, 3), device=dev), tgt=torch.empty((F * P1,), device=dev),
                  grad_host=[torch.empty_like(x).pin_memory() for x in host],
                  loss_host=torch.empty((), dtype=torch.float32).pin_memory())
             for _ in range(2)]

    def prefetch(i):
        sl = slots[i % 2]
        k = i % len(renderers)
        s = k * F
        with torch.cuda.stream(copy_stream):
            copy_stream.wait_event(sl["free"])
            for d, x in zip(sl["ps"], host):
                d.copy_(x, non_blocking=True)
            sl["pix"].copy_(sweep_pix[s * P1:(s + F) * P1], non_blocking=True)
            sl["tgt"].copy_(tgt_host[s * P1:(s + F) * P1], non_blocking=True)
            sl["ready"].record(copy_stream)
        sl["step"] = i

    def step(i):
        sl = slots[i % 2]
        sl["landed"].synchronize()  # step i-2's loss and gradients are on the host
        sl["outs"] = None  # ... so its device results can be recycled
        if sl["step"] != i:
            prefetch(i)
        compute.wait_event(sl["ready"])
        pix, tgt = sl["pix"], sl["tgt"]
        prefetch(i + 1)
        ps = [x.detach().requires_grad_(True) for x in sl["ps"]]
        img, alpha, depth = renderers[i % len(renderers)](*ps, pix)
        loss = (img - tgt).abs().mean()
        loss.backward()
        outs = [loss.detach()] + [p.grad for p in ps]
        done = torch.cuda.Event()
        done.record(compute)
        with torch.cuda.stream(d2h_stream):
            d2h_stream.wait_event(done)
            sl["loss_host"].copy_(outs[0], non_blocking=True)
            for gh, g in zip(sl["grad_host"], outs[1:]):
                gh.copy_(g, non_blocking=True)
            sl["landed"].record(d2h_stream)
        sl["outs"] = outs  # kept until the copies have landed (no cross-stream frees)
        sl["free"].record(compute)

    def timed_e2e(steps, warm):
        for i in range(warm):
            step(i)
        compute.wait_stream(d2h_stream)
        timed_barrier()
        st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m0 = torch.cuda.memory_stats(dev)
        st.record(compute)
        for i in range(steps):
            step(warm + i)
        compute.wait_stream(d2h_stream)  # the last step's results have reached the host
        en.record(compute)
        m1 = torch.cuda.memory_stats(dev)
        timed_barrier()
        allocs = {k: int(m1.get(k, 0) - m0.get(k, 0)) for k in ("num_device_alloc", "num_device_free",
                                                                  "num_alloc_retries")}
        return max_over_ranks(st.elapsed_time(en), device=dev), allocs

    # pinned-memory copy bandwidth of this machine, one transfer of a step's inputs each way
    probe = torch.empty(sum(x.numel() for x in host) + 2 * F * P1 * 4, dtype=torch.float32).pin_memory()
    probe_dev = torch.empty(probe.shape, dtype=torch.float32, device=dev)
    link = {}
    for name, dst, src in (("h2d", probe_dev, probe), ("d2h", probe, probe_dev)):
        dst.copy_(src, non_blocking=True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        dst.copy_(src, non_blocking=True)
        e1.record()
        e1.synchronize()
        link[name] = round(probe.numel() * 4 / (e0.elapsed_time(e1) / 1e3) / 1e9, 1)
    del probe, probe_dev

    # priming: one synchronised call per renderer fixes the instance capacity
    cap = 0
    for k, r in enumerate(renderers):
        step(k)
        cap = max(cap, int(r.last["binning"].capacity), int(r.last["binning"].total * 1.25) + 1024)
    for r in renderers:
        r.params["capacity"] = cap
        r.params["sync_check"] = False
    ms, alloc = timed_e2e(a.steps, a.warmup)
    for r in renderers:
        if "binning" in r.last:
            total, flags = UG.read_status(r.last["binning"])
            if flags:
                raise RuntimeError(f"e2e: binning flags {flags} (instances {total}, capacity {cap})")
    h2d = sum(x.numel() * x.element_size() for x in host) + F * P1 * 3 * 4 + F * P1 * 4
    d2h = 4 + sum(x.numel() * x.element_size() for x in host)
    return {"value": round(a.steps * F * world / (ms / 1e3), 3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "api": "us3d_b200.batch.UltraGaussBatchRenderer (autograd)",
            "copies": "next step's inputs prefetched on a second stream (double buffered); results read back on a "
                      "third stream; the host waits for step i-2's results before launching step i",
            "pinned_copy_gbs": link, "device_allocations_in_timed_steps": alloc}


def cpu_baseline(a, sc, specs, frames: int = 1):
    """The C oracle (restatement of the reference algorithm) on the host cores, on a bounded
    sample: `frames` full frames of the same workload (mapper + forward + backward)."""
    import numpy as np

    from oracle import ultragauss_oracle as O

    nt = os.cpu_count() or 1
    O.set_threads(nt)
    means, tril = sc.means.numpy(), sc.precision_tril.numpy()
    op, it = sc.opacities.numpy(), sc.intensities.numpy()
    t0 = time.perf_counter()
    for f in range(frames):
        s = specs[f]
        from us3d_b200 import scenes

        pix = scenes.slice_pixels(s.origin, s.axis_lat, s.axis_ax, s.height, s.width, s.lateral_spacing,
                                  s.axial_spacing, s.axial_near, s.lateral_col_offset).numpy()
        geo = O.geometry(s.origin, s.axis_lat, s.axis_ax, s.axis_ele, s.lateral_spacing, s.axial_spacing,
                         s.axial_near, s.lateral_col_offset)
        st = O.render(means, tril, op, it, pix, geo, s.height, s.width, 7.815, 1e-4, True, 1e-6, 0.0,
                      want_ambiguous=False)
        rng = np.random.default_rng(f)
        dI = np.sign(st["image"] - rng.random(st["image"].shape[0]).astype(np.float32)) / st["image"].shape[0]
        z = np.zeros_like(dI)
        O.backward(st, dI, z, z)
    dt = time.perf_counter() - t0
    return {"value": round(frames / dt, 5), "unit": UNIT, "cores": nt, "kind": "port",
            "sample": f"{frames} full frame(s) of the workload ({a.gaussians} Gaussians, {a.size}^2 px): "
                      f"C oracle mapper + per-pixel candidate lists + forward + backward, {dt:.1f} s"}


def cpu_baseline_dense(frames: int = 2):
    """The reference's own CPU path for UltraGauss (its dense PyTorch fallback, restated in
    oracle/ultragauss_dense_fallback.py) with autograd backward and an L1 loss, on all host
    threads, at the survey's config-1 size (4,096 Gaussians, 128x128 frames at 0.3 mm):
    `frames` frames are timed."""
    import torch

    from oracle.ultragauss_dense_fallback import render_dense
    from us3d_b200 import scenes

    nt = os.cpu_count() or 1
    torch.set_num_threads(nt)
    sc = scenes.make_scene(4096, seed=0)
    sweep = scenes.linear_sweep(16, 128, 128, 0.3, seed=0)
    ps = [sc.means.clone(), sc.precision_tril.clone(),
          torch.logit(sc.opacities.clamp(1e-6, 1 - 1e-6)).reshape(-1, 1),
          torch.logit(sc.intensities.clamp(1e-6, 1 - 1e-6)).reshape(-1, 1)]
    ps = [p.requires_grad_(True) for p in ps]
    tgt = torch.rand((16, 128 * 128), generator=torch.Generator().manual_seed(1))
    t0 = time.perf_counter()
    for f in range(frames):
        img, _ = render_dense(*ps, sweep[f].pixels, 1e-4, 128, 128)
        loss = (img.reshape(-1) - tgt[f]).abs().mean()
        loss.backward()
    dt = time.perf_counter() - t0
    return {"value": round(frames / dt, 4), "unit": UNIT, "cores": nt, "kind": "port",
            "sample": f"{frames} frames at config-1 size (4096 Gaussians, 128^2 px): the reference's dense PyTorch "
                      f"CPU fallback (restated) + autograd backward, {dt:.1f} s"}


def reference_cuda(a, sc, specs, frames: int = 8, warm: int = 2):
    """The reference's own UltraGauss CUDA (its sources built for sm_100a into oracle/_ref)
    on this box's GPU, one frame per call as its pipeline renders: mapper, forward and
    backward of each frame with an L1 upstream gradient, timed with CUDA events on the
    current stream (the reference's host synchronisations inside each call included)."""
    import torch

    ref_dir = ROOT / "oracle" / "_ref"
    if not torch.cuda.is_available() or not any(ref_dir.glob("ultragauss_ref_C*.so")):
        return {"unavailable": "no GPU or no reference build in oracle/_ref"}
    sys.path.insert(0, str(ref_dir))
    import ultragauss_ref_C as REF

    from us3d_b200 import scenes

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    pad = lambda x: torch.nn.functional.pad(x, (0, 1)).contiguous()  # noqa: E731
    mp = pad(sc.means.to(dev))
    tril = sc.precision_tril.to(dev).contiguous()
    attr = torch.stack([sc.opacities, sc.intensities], 1).to(dev).contiguous()
    g = torch.Generator().manual_seed(5)
    inputs = []
    for s in specs[:max(1, min(frames, len(specs)))]:
        v = lambda x: torch.as_tensor(x, dtype=torch.float32).to(dev).contiguous()  # noqa: E731
        pix = scenes.slice_pixels(s.origin, s.axis_lat, s.axis_ax, s.height, s.width, s.lateral_spacing,
                                  s.axial_spacing, s.axial_near, s.lateral_col_offset)
        tgt = torch.rand((s.height * s.width,), generator=g).to(dev)
        inputs.append((s, pad(pix.to(dev)), v(s.origin), v(s.axis_lat), v(s.axis_ax), v(s.axis_ele), tgt))

    def frame(i):
        s, pp, o, l, ax, e, tgt = inputs[i % len(inputs)]
        counts, offsets, indices = REF.MapperForwardCUDA(pp, mp, tril, o, l, ax, e, s.height, s.width,
                                                         s.lateral_spacing, s.axial_spacing, s.axial_near,
                                                         s.lateral_col_offset, 7.815, True, 1e-4)
        image, alpha, depth, sic = REF.ShaderForwardCUDA(attr, mp, tril, pp, o, e, offsets, counts, indices, 1e-6,
                                                         0.0, 7.815, 1e-4)
        dI = torch.sign(image.reshape(-1) - tgt) / tgt.numel()
        z = torch.zeros_like(dI)
        REF.ShaderBackwardCUDA(dI, z, z, attr, mp, tril, pp, o, e, offsets, counts, indices, sic, alpha, 1e-6, 0.0,
                               7.815, 1e-4)

    for i in range(warm):
        frame(i)
    torch.cuda.synchronize()
    st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st.record()
    for i in range(frames):
        frame(i)
    en.record()
    en.synchronize()
    ms = st.elapsed_time(en)
    return {"value": round(frames / (ms / 1e3), 3), "unit": UNIT, "frames": frames, "ms_per_frame": round(ms / frames, 3),
            "kind": "the reference's own UltraGauss CUDA (MapperForwardCUDA + ShaderForwardCUDA + ShaderBackwardCUDA), "
                    "built for sm_100a from its sources, one frame per call, CUDA events on the current stream"}


def run_reference(a):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import torch  # noqa: F401

    from us3d_b200 import scenes
    from us3d_b200 import ultragauss as UG

    sc = scenes.make_scene(a.gaussians, seed=0)
    sweep = scenes.linear_sweep(max(a.steps + a.warmup, 1), a.size, a.size, a.spacing, seed=0)
    specs = [UG.SliceSpec(f.height, f.width, f.lateral_spacing, f.axial_spacing, f.axial_near, f.lateral_col_offset,
                          f.origin, f.axis_lat, f.axis_ax, f.axis_ele) for f in sweep]
    if a.warmup:  # the oracle has no warm-up state; one untimed frame pages its code in
        cpu_baseline(a, sc, specs[:1], frames=1)
    times = []
    for i in range(a.steps):
        r = cpu_baseline(a, sc, [specs[i % len(specs)]], frames=1)
        times.append(1.0 / r["value"])
    value = a.steps / sum(times)
    cb = {"value": round(value, 5), "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
          "sample": f"{a.steps} step(s) of 1 full frame each ({a.gaussians} Gaussians, {a.size}^2 px): C restatement "
                    "of the reference UltraGauss mapper + forward + backward on all host threads"}
    # one frame per step: the reference renders one frame per call
    cfg = workload_config(a, 1)
    cfg["frames_per_step"] = 1
    cfg["workload"] = cfg["workload"].replace(f"{a.frames_per_step} frames/step per GPU", "1 frame per step")
    out = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": world, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": round(1e3 * sum(times) / a.steps, 2), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic: seeded headline scene",
           "config": cfg, "impl": "reference", "cpu_baseline": cb,
           "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    try:
        out["reference_cuda"] = reference_cuda(a, sc, specs)
    except Exception as ex:  # the CPU arm stands on its own; say why the GPU number is missing
        out["reference_cuda"] = {"unavailable": f"{type(ex).__name__}: {ex}"[:300]}
    print(json.dumps(out), flush=True)


def relaunch_multi_gpu(a) -> int:
    """`python bench.py --gpus N` outside a launcher: start N ranks (one per GPU) with
    torch.distributed.run on this node, each running this script with the same arguments,
    and return its exit status. Frames are sharded across the ranks (replicas, no collective
    on the data path); rank 0 prints the line."""
    import socket

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={a.gpus}",
           "--master-addr=127.0.0.1", f"--master-port={port}", str(Path(__file__).resolve()), *sys.argv[1:]]
    return subprocess.call(cmd)


def main():
    a = parse()
    if a.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(relaunch_multi_gpu(a))
    if a.impl == "reference":
        run_reference(a)
    else:
        run_b200(a)


if __name__ == "__main__":
    main()
