"""Batched UltraGauss rendering: many frames of any sizes in one launch sequence.

``UltraGaussBatchRenderer(frames)(means, precision_tril, opacities, intensities, pixels)``
renders every frame of ``frames`` (a list of ``SliceSpec``) in one binning + one forward
launch and returns concatenated (image, alpha, depth) over all frames' pixels; its
backward runs one adjoint launch and returns gradients summed over the frames. This is
the batched form of the reference's per-frame UltraGaussRenderer (one frame per call).
"""

from __future__ import annotations

from typing import Optional, Sequence

import torch

from . import ultragauss as UG


class _BatchFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, frames: UG.FrameTable, params: dict, means, tril, opac, inten, pixels, holder):
        want_counts = params.get("want_counts", False)
        cull = params.get("slice_cull", True) and not want_counts
        b = UG.bin_gaussians(means, tril, opac, inten, frames, params["chi2"], params["beta"], params["sort_by_depth"],
                             capacity=params.get("capacity"), sync_check=params.get("sync_check", True),
                             slice_cull_pixels=pixels if cull else None)
        image, alpha, depth, counts = UG.forward(b, pixels, params["bg_alpha"], params["bg_intensity"],
                                                 want_counts=params.get("want_counts", False))
        ctx.b = b
        ctx.params = params
        ctx.save_for_backward(pixels, alpha)
        if holder is not None:
            holder["binning"] = b
            holder["counts"] = counts
        return image, alpha, depth

    @staticmethod
    def backward(ctx, d_image, d_alpha, d_depth):
        pixels, alpha = ctx.saved_tensors
        p = ctx.params
        dm, dt, do, di = UG.backward(ctx.b, pixels, d_image.contiguous(), d_alpha.contiguous(), d_depth.contiguous(),
                                     alpha, p["bg_alpha"], p["bg_intensity"])
        return None, None, dm, dt, do, di, None, None


class UltraGaussBatchRenderer:
    def __init__(self, frames: Sequence[UG.SliceSpec], device: torch.device, chi2_threshold: float = 7.815,
                 diag_beta: float = 1e-4, mapper_sort_by_depth: bool = True, fixed_bg_alpha: float = 1e-6,
                 fixed_bg_intensity: float = 0.0, capacity: Optional[int] = None, slice_cull: bool = True):
        self.frames = UG.build_frame_table(list(frames), device)
        self.params = dict(chi2=float(chi2_threshold), beta=float(diag_beta), sort_by_depth=bool(mapper_sort_by_depth),
                           bg_alpha=float(fixed_bg_alpha), bg_intensity=float(fixed_bg_intensity), capacity=capacity,
                           slice_cull=bool(slice_cull))
        self.last = {}

    @property
    def n_pixels(self) -> int:
        return self.frames.n_pixels

    def __call__(self, means, precision_tril, opacities, intensities, pixels):
        self.last = {}
        return _BatchFunction.apply(self.frames, self.params, means, precision_tril.contiguous(),
                                    opacities.reshape(-1), intensities.reshape(-1), pixels, self.last)


class GraphedTrainingStep:
    """One training step of a batch of frames, captured once as a CUDA graph and replayed.

    The step is: bin (slice-culled, fixed instance capacity, no host readback), forward,
    ``loss_grad(image, alpha, depth) -> (d_image, d_alpha, d_depth)`` (any stream-ordered
    PyTorch code), backward into the static gradient buffers ``grads``. Parameters, pixel
    positions and whatever ``loss_grad`` reads must stay at the same addresses between
    replays (update them in place). The capacity is set from a synchronised priming binning
    times ``margin``; ``check()`` reads the last replay's flags (one synchronisation) and
    raises if the instances outgrew it, after which the step should be rebuilt."""

    def __init__(self, frames: Sequence[UG.SliceSpec], device: torch.device, params, pixels, loss_grad,
                 grads=None, chi2_threshold: float = 7.815, diag_beta: float = 1e-4, sort_by_depth: bool = True,
                 bg_alpha: float = 1e-6, bg_intensity: float = 0.0, margin: float = 1.25):
        self.frames = UG.build_frame_table(list(frames), device)
        self.params = [params[0], params[1].contiguous(), params[2].reshape(-1), params[3].reshape(-1)]
        self.pixels = pixels
        self.loss_grad = loss_grad
        self.cfg = (float(chi2_threshold), float(diag_beta), bool(sort_by_depth))
        self.bg = (float(bg_alpha), float(bg_intensity))
        G = self.params[0].shape[0]
        self.grads = grads if grads is not None else (
            torch.empty((G, 3), device=device), torch.empty((G, 6), device=device), torch.empty((G,), device=device),
            torch.empty((G,), device=device))
        prime = UG.bin_gaussians(*self.params, self.frames, *self.cfg, slice_cull_pixels=pixels)
        # at least the capacity the priming binning succeeded with: with many small frames the
        # (Gaussian, frame) pairs, which the capacity also bounds, can outnumber a quarter of it
        self.capacity = max(int(prime.capacity), int(prime.total * margin) + 1024)
        self.binning = None
        self._run()  # uncaptured: sets kernel attributes and allocator state
        torch.cuda.synchronize(device)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._run()

    def _run(self):
        b = UG.bin_gaussians(*self.params, self.frames, *self.cfg, capacity=self.capacity, sync_check=False,
                             slice_cull_pixels=self.pixels)
        image, alpha, depth, _ = UG.forward(b, self.pixels, *self.bg, want_counts=False)
        d_image, d_alpha, d_depth = self.loss_grad(image, alpha, depth)
        UG.backward(b, self.pixels, d_image.contiguous(), d_alpha.contiguous(), d_depth.contiguous(), alpha, *self.bg,
                    out=self.grads)
        self.binning = b
        self.outputs = (image, alpha, depth)

    def replay(self):
        self.graph.replay()
        return self.grads

    def check(self):
        total, flags = UG.read_status(self.binning)
        if flags:
            raise RuntimeError(f"graphed step: binning flags {flags} ({total} instances, capacity {self.capacity})")
        return total


LAUNCH_SHAPES = [(b, t) for b in (128, 256, 512) for t in (128, 256)]
BACKWARD_VARIANTS = (0, 1)  # one pixel per FP32 instruction / two pixels per packed FP32 pair
FORWARD_VARIANTS = (0, 1)   # one pixel per thread / two pixels per thread in packed FP32 pairs


def get_forward_variant() -> int:
    import ctypes

    from . import _lib

    v = ctypes.c_int32(0)
    _lib.check(_lib.call("us3d_ug_get_forward_variant", ctypes.byref(v)), "us3d_ug_get_forward_variant")
    return int(v.value)


def set_forward_variant(variant: int) -> None:
    from . import _lib

    _lib.check(_lib.call("us3d_ug_set_forward_variant", int(variant)), "us3d_ug_set_forward_variant")


def get_backward_variant() -> int:
    import ctypes

    from . import _lib

    v = ctypes.c_int32(0)
    _lib.check(_lib.call("us3d_ug_get_backward_variant", ctypes.byref(v)), "us3d_ug_get_backward_variant")
    return int(v.value)


def set_backward_variant(variant: int) -> None:
    from . import _lib

    _lib.check(_lib.call("us3d_ug_set_backward_variant", int(variant)), "us3d_ug_set_backward_variant")


def get_launch_config():
    """(forward batch, backward threads) the UltraGauss shading kernels launch with."""
    import ctypes

    from . import _lib

    fb, bt = ctypes.c_int32(0), ctypes.c_int32(0)
    _lib.check(_lib.call("us3d_ug_get_launch_config", ctypes.byref(fb), ctypes.byref(bt)), "us3d_ug_get_launch_config")
    return int(fb.value), int(bt.value)


def set_launch_config(forward_batch: int, backward_threads: int) -> None:
    from . import _lib

    _lib.check(_lib.call("us3d_ug_set_launch_config", int(forward_batch), int(backward_threads)),
               "us3d_ug_set_launch_config")


def autotune_launch(frames: UG.FrameTable, params, pixels: torch.Tensor, reps: int = 3,
                    chi2_threshold: float = 7.815, diag_beta: float = 1e-4, bg_alpha: float = 1e-6):
    """Times the batched step (slice-culled bin, forward, backward with a seeded upstream
    gradient) on the caller's frames for every launch shape the library is built for and every
    forward and backward variant, keeps the fastest (set_launch_config, set_backward_variant,
    set_forward_variant) and returns {(forward_batch, backward_threads, backward_variant,
    forward_variant): ms per step}. Neither the shapes nor the forward variants change any
    result; the backward variants differ in summation order only. Synchronises; run it before
    capturing graphs."""
    means, tril, opac, inten = params[0], params[1].contiguous(), params[2].reshape(-1), params[3].reshape(-1)
    g = torch.Generator(device=pixels.device)
    g.manual_seed(0)
    d_image = torch.randn(frames.n_pixels, generator=g, device=pixels.device)
    zeros = torch.zeros_like(d_image)
    b = UG.bin_gaussians(means, tril, opac, inten, frames, chi2_threshold, diag_beta, True,
                         slice_cull_pixels=pixels)
    cap = b.capacity

    def step():
        bb = UG.bin_gaussians(means, tril, opac, inten, frames, chi2_threshold, diag_beta, True, capacity=cap,
                              sync_check=False, slice_cull_pixels=pixels)
        img, alpha, depth, _ = UG.forward(bb, pixels, bg_alpha, 0.0, want_counts=False)
        UG.backward(bb, pixels, d_image, zeros, zeros, alpha, bg_alpha, 0.0)

    timings = {}
    for fvariant in FORWARD_VARIANTS:
        set_forward_variant(fvariant)
        for variant in BACKWARD_VARIANTS:
            set_backward_variant(variant)
            for shape in LAUNCH_SHAPES:
                if fvariant == 1 and shape[0] == 512:
                    continue  # the packed forward stages at most 256 Gaussians (same as 256)
                set_launch_config(*shape)
                step()
                torch.cuda.synchronize(pixels.device)
                st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                st.record()
                for _ in range(reps):
                    step()
                en.record()
                en.synchronize()
                timings[(*shape, variant, fvariant)] = st.elapsed_time(en) / reps
    best = min(timings, key=timings.get)
    set_launch_config(best[0], best[1])
    set_backward_variant(best[2])
    set_forward_variant(best[3])
    return timings
