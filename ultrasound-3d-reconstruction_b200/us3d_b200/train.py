"""The training step around the UltraGauss renderer, on the device in a handful of launches.

The reference trains with PyTorch around its renderer (pipeline_god_file.py:727-767): per
step, ``GaussianParameters`` activates the raw parameters (opacities and intensities through
``torch.sigmoid``, pipeline_god_file.py:368-372; means and the raw precision factor are used
as they are, :494), the renderer runs forward, ``image_loss`` (L1 + optional global SSIM,
:606-637) gives the loss, autograd runs the renderer's backward and the activations'
backward, and ``torch.optim.Adam`` (lr 1e-3, :740) updates every parameter. Here the same step
is: binning with the logistic activation folded into its parameter packing, forward, the
per-frame loss reduced to gradient coefficients (``us3d_ug_loss``), the backward with the loss
gradient computed inside its pixel staging (``us3d_ug_backward_loss``), and one multi-tensor
Adam launch that also applies the activation's chain rule (``us3d_adam_step``). A batch of F
frames is trained on the sum of its frames' losses (each frame keeps the gradient of a
single-frame step). ``UltraGaussTrainer`` captures the step as a CUDA graph.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional, Sequence

import torch

from . import _lib
from . import ultragauss as UG
from .ultragauss import _ptr, _stream


@dataclass
class TrainConfig:
    """Defaults of the reference's GodConfig for UltraGauss training (pipeline_god_file.py:
    89-122) and of its render settings (baselines/ultragauss/render.py:61-62)."""

    lr: float = 1.0e-3
    beta1: float = 0.9
    beta2: float = 0.999
    eps: float = 1.0e-8
    l1_weight: float = 1.0
    ssim_weight: float = 0.0
    chi2_threshold: float = 7.815
    diag_beta: float = 1.0e-4
    sort_by_depth: bool = True
    bg_alpha: float = 1.0e-6
    bg_intensity: float = 0.0


def _logit(x: torch.Tensor) -> torch.Tensor:
    x = x.clamp(1.0e-6, 1.0 - 1.0e-6)
    return torch.log(x / (1.0 - x))


class UltraGaussParameters:
    """The raw parameters the reference's training loop optimises for UltraGauss (the fields of
    GaussianParameters that reach the renderer, pipeline_god_file.py:340-372): means (G,3),
    raw_precision_tril (G,6), raw_opacities (G,1) and raw_intensities (G,1), both logits."""

    def __init__(self, means: torch.Tensor, raw_precision_tril: torch.Tensor, raw_opacities: torch.Tensor,
                 raw_intensities: torch.Tensor):
        G = means.shape[0]
        self.means = means.float().contiguous()
        self.raw_precision_tril = raw_precision_tril.float().contiguous()
        self.raw_opacities = raw_opacities.float().reshape(G, 1).contiguous()
        self.raw_intensities = raw_intensities.float().reshape(G, 1).contiguous()

    @classmethod
    def from_points(cls, init_means: torch.Tensor, init_intensities: torch.Tensor, init_scale_mm: float = 0.5,
                    init_opacity: float = 0.1, diag_beta: float = 1.0e-4) -> "UltraGaussParameters":
        """The reference's initialisation (GaussianParameters.__init__ and _init_precision_tril,
        pipeline_god_file.py:344-390): isotropic raw factor sqrt(max(1/s - beta, 1e-4)) on the
        diagonal, opacity logit(init_opacity), intensity logit(clamp(init, 1e-4, 1 - 1e-4))."""
        n = init_means.shape[0]
        dev = init_means.device
        raw_diag = math.sqrt(max(1.0 / max(float(init_scale_mm), 1.0e-4) - float(diag_beta), 1.0e-4))
        tril = torch.zeros((n, 6), device=dev)
        tril[:, 0] = raw_diag
        tril[:, 3] = raw_diag
        tril[:, 5] = raw_diag
        return cls(init_means.float(), tril, _logit(torch.full((n, 1), float(init_opacity), device=dev)),
                   _logit(init_intensities.float().reshape(n, 1).clamp(1.0e-4, 1.0 - 1.0e-4)))

    def tensors(self) -> List[torch.Tensor]:
        return [self.means, self.raw_precision_tril, self.raw_opacities, self.raw_intensities]

    def opacities(self) -> torch.Tensor:
        return torch.sigmoid(self.raw_opacities)

    def intensities(self) -> torch.Tensor:
        return torch.sigmoid(self.raw_intensities)


class Adam:
    """torch.optim.Adam (no weight decay, no amsgrad) over a list of float32 tensors, one
    launch per step. ``logistic[i]`` marks tensor i as logits whose gradient is given w.r.t.
    their logistic activation (the chain rule is applied in the update)."""

    def __init__(self, params: Sequence[torch.Tensor], lr: float = 1.0e-3, betas=(0.9, 0.999), eps: float = 1.0e-8,
                 logistic: Optional[Sequence[bool]] = None):
        if len(params) > _lib.ADAM_MAX_TENSORS:
            raise ValueError(f"at most {_lib.ADAM_MAX_TENSORS} tensors per Adam launch")
        for p in params:
            if p.dtype != torch.float32 or not p.is_contiguous():
                raise ValueError("Adam tensors must be contiguous float32")
        self.params = list(params)
        self.exp_avg = [torch.zeros_like(p) for p in self.params]
        self.exp_avg_sq = [torch.zeros_like(p) for p in self.params]
        self.lr, self.betas, self.eps = float(lr), (float(betas[0]), float(betas[1])), float(eps)
        self.logistic = list(logistic) if logistic is not None else [False] * len(self.params)
        self.step_count = 0

    def step(self, grads: Sequence[torch.Tensor], step: Optional[int] = None) -> None:
        """One update with ``grads`` (same shapes as the parameters; read, not modified)."""
        self.step_count = self.step_count + 1 if step is None else int(step)
        table = (_lib.AdamTensor * len(self.params))()
        for i, (p, g, m, v) in enumerate(zip(self.params, grads, self.exp_avg, self.exp_avg_sq)):
            if g.numel() != p.numel() or not g.is_contiguous():
                raise ValueError(f"gradient {i}: expected {p.numel()} contiguous elements")
            table[i] = _lib.AdamTensor(_ptr(p), _ptr(g), _ptr(m), _ptr(v), p.numel(),
                                       _lib.ADAM_LOGISTIC if self.logistic[i] else _lib.ADAM_IDENTITY, 0)
        _lib.check(_lib.call("us3d_adam_step", table, len(self.params), self.lr, self.betas[0], self.betas[1],
                             self.eps, self.step_count, _stream()), "us3d_adam_step")


class UltraGaussTrainer:
    """Training steps on fixed batches of frames: slice-culled binning (logistic activation
    folded in) -> forward -> per-frame loss -> backward with the fused loss gradient, replayed
    from one CUDA graph per batch, then Adam on all four parameter tensors (one launch).

    ``batches`` is a list of (frame specs or a FrameTable, pixel positions (P,3), targets (P,))
    on the device; frame tables, pixel positions and targets must stay at their addresses
    (refresh them in place). The instance capacity of each batch is fixed from a synchronised
    priming binning times ``margin``; ``check()`` reads the flags of every batch's last replay
    (one synchronisation per batch) and raises if a binning outgrew its capacity. ``losses()``
    returns the last replay's per-frame statistics (synchronises). ``from_source`` trains on
    random batches drawn on the device from a ``frames.DeviceFrameSource``. With ``refine``
    (a refine.RefineConfig) the Gaussians are densified and pruned on its schedule: the
    statistics are accumulated on the device every step, and after a refinement the parameter
    and gradient buffers are new, so every batch's graph is captured again and its instance
    capacity primed again (``refine_log`` lists the counts of each refinement)."""

    def __init__(self, params: UltraGaussParameters, batches, cfg: Optional[TrainConfig] = None,
                 margin: float = 1.25, graph: bool = True, refine=None):
        self.params = params
        self.cfg = cfg or TrainConfig()
        self.margin = float(margin)
        self.refine_cfg = refine
        self.refine_log = []
        dev = params.means.device
        G = params.means.shape[0]
        self.grads = (torch.empty((G, 3), device=dev), torch.empty((G, 6), device=dev), torch.empty((G,), device=dev),
                      torch.empty((G,), device=dev))
        self.optimizer = Adam(params.tensors(), self.cfg.lr, (self.cfg.beta1, self.cfg.beta2), self.cfg.eps,
                              logistic=[False, False, True, True])
        self._batches = []
        self.source = None
        for specs, pixels, targets in batches:
            frames = specs if isinstance(specs, UG.FrameTable) else UG.build_frame_table(list(specs), dev)
            prime = UG.bin_gaussians(*self._render_args(), frames, self.cfg.chi2_threshold, self.cfg.diag_beta,
                                     self.cfg.sort_by_depth, slice_cull_pixels=pixels, logit_attributes=True)
            cap = max(int(prime.capacity), int(prime.total * margin) + 1024)
            self._batches.append(dict(frames=frames, pixels=pixels, targets=targets, capacity=cap, binning=None,
                                      stats=torch.zeros((frames.n_frames, 8), dtype=torch.float64, device=dev),
                                      coef=torch.zeros((frames.n_frames, 4), device=dev), graph=None))
        self.graph = graph
        self.steps_done = 0
        self.refine_stats = None
        if refine is not None:
            from .refine import RefineStats

            self.refine_stats = RefineStats(G, dev)
            self.refine_gen = torch.Generator(device=dev)
            self.refine_gen.manual_seed(0)

    @classmethod
    def from_source(cls, params: UltraGaussParameters, source, batch_size: int, cfg: Optional[TrainConfig] = None,
                    margin: float = 1.5, prime_batches: int = 4, seed: int = 0, graph: bool = True,
                    indices: Optional[torch.Tensor] = None, refine=None) -> "UltraGaussTrainer":
        """Trains on batches of ``batch_size`` frames of ``source`` (a DeviceFrameSource): each
        step draws dataset indices on the device (uniformly among ``indices``, all frames by
        default; the reference draws one frame per step with np.random.choice) and assembles the
        batch in place with one launch. The instance capacity is the largest of
        ``prime_batches`` random batches times ``margin``."""
        dev = source.device
        pool = (indices if indices is not None else torch.arange(source.n)).to(dev, torch.int64)
        gen = torch.Generator(device=dev)
        gen.manual_seed(int(seed))
        table = source.frame_table(batch_size)
        hw = source.height * source.width
        pixels = torch.empty((batch_size * hw, 3), device=dev)
        targets = torch.empty((batch_size * hw,), device=dev)
        draw = torch.empty((batch_size,), dtype=torch.int64, device=dev)
        c = cfg or TrainConfig()
        best = worked = 0
        for _ in range(max(1, int(prime_batches))):
            torch.randint(0, pool.numel(), (batch_size,), generator=gen, device=dev, out=draw)
            source.fill(pool[draw], table, pixels, targets)
            b = UG.bin_gaussians(params.means, params.raw_precision_tril, params.raw_opacities.reshape(-1),
                                 params.raw_intensities.reshape(-1), table, c.chi2_threshold, c.diag_beta,
                                 c.sort_by_depth, slice_cull_pixels=pixels, logit_attributes=True)
            best = max(best, b.total)
            worked = max(worked, int(b.capacity))
        self = cls(params, [(table, pixels, targets)], c, margin=1.0, graph=graph, refine=refine)
        self._batches[0]["capacity"] = max(worked, int(best * margin) + 1024)
        self.source = dict(source=source, pool=pool, gen=gen, draw=draw, prime_batches=max(1, int(prime_batches)),
                           margin=float(margin))
        return self

    def _render_args(self):
        p = self.params
        return p.means, p.raw_precision_tril, p.raw_opacities.reshape(-1), p.raw_intensities.reshape(-1)

    def _forward_backward(self, bt) -> None:
        c = self.cfg
        b = UG.bin_gaussians(*self._render_args(), bt["frames"], c.chi2_threshold, c.diag_beta, c.sort_by_depth,
                             capacity=bt["capacity"], sync_check=False, slice_cull_pixels=bt["pixels"],
                             logit_attributes=True)
        image, alpha, depth, _ = UG.forward(b, bt["pixels"], c.bg_alpha, c.bg_intensity, want_counts=False)
        UG.loss(bt["frames"], image, bt["targets"], c.l1_weight, c.ssim_weight, out=(bt["stats"], bt["coef"]))
        UG.backward_loss(b, bt["pixels"], image, bt["targets"], bt["coef"], alpha, c.bg_alpha, c.bg_intensity,
                         out=self.grads)
        bt["binning"] = b
        bt["image"] = image

    def step(self, batch_index: int = 0) -> None:
        """One training step on batch ``batch_index``: forward + loss + backward (replayed from
        a CUDA graph once captured) and the Adam update (one launch; its step count and bias
        corrections change every step, so it runs outside the graph)."""
        bt = self._batches[batch_index]
        if self.source is not None:
            sc = self.source
            torch.randint(0, sc["pool"].numel(), sc["draw"].shape, generator=sc["gen"], device=sc["draw"].device,
                          out=sc["draw"])
            sc["source"].fill(sc["pool"][sc["draw"]], bt["frames"], bt["pixels"], bt["targets"])
        if not self.graph:
            self._forward_backward(bt)
        elif bt["graph"] is None:
            self._forward_backward(bt)  # uncaptured first run: kernel attributes, allocator state
            torch.cuda.synchronize(self.params.means.device)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._forward_backward(bt)
            bt["graph"] = g
            g.replay()
        else:
            bt["graph"].replay()
        self.optimizer.step(self.grads)
        self.steps_done += 1
        if self.refine_stats is not None:
            self.refine_stats.accumulate(self.grads[0])
            if self.refine_cfg.due(self.steps_done):
                self._refine()

    def _refine(self) -> None:
        from .refine import refine

        self.refine_log.append(dict(step=self.steps_done, **refine(self.params, self.optimizer, self.refine_stats,
                                                                    self.refine_cfg, self.refine_gen)))
        self._rebuffer()

    def _rebuffer(self) -> None:
        """New gradient buffers, graphs and instance capacities after the parameter tensors were
        replaced (a refinement or a loaded checkpoint with another number of Gaussians)."""
        dev = self.params.means.device
        G = self.params.means.shape[0]
        self.grads = (torch.empty((G, 3), device=dev), torch.empty((G, 6), device=dev),
                      torch.empty((G,), device=dev), torch.empty((G,), device=dev))
        c = self.cfg
        for bt in self._batches:
            bt["graph"] = None  # parameter and gradient buffers moved: capture again
            bt["binning"] = None
            if self.source is None:
                prime = UG.bin_gaussians(*self._render_args(), bt["frames"], c.chi2_threshold, c.diag_beta,
                                         c.sort_by_depth, slice_cull_pixels=bt["pixels"], logit_attributes=True)
                bt["capacity"] = max(int(prime.capacity), int(prime.total * self.margin) + 1024)
        if self.source is not None:
            sc, bt = self.source, self._batches[0]
            best = worked = 0
            for _ in range(sc["prime_batches"]):
                torch.randint(0, sc["pool"].numel(), sc["draw"].shape, generator=sc["gen"], device=dev, out=sc["draw"])
                sc["source"].fill(sc["pool"][sc["draw"]], bt["frames"], bt["pixels"], bt["targets"])
                prime = UG.bin_gaussians(*self._render_args(), bt["frames"], c.chi2_threshold, c.diag_beta,
                                         c.sort_by_depth, slice_cull_pixels=bt["pixels"], logit_attributes=True)
                best = max(best, prime.total)
                worked = max(worked, int(prime.capacity))
            bt["capacity"] = max(worked, int(best * sc["margin"]) + 1024)

    _PARAM_NAMES = ("means", "raw_precision_tril", "raw_opacities", "raw_intensities")

    def state_dict(self) -> dict:
        """Everything a resumed run needs, as the reference's checkpoint (config, iteration,
        parameters, optimizer state; pipeline_god_file.py:701-724) plus the refinement
        statistics and log and the generators of the batch draws and the refinement: a run
        resumed from it takes the same steps, bit for bit, as the uninterrupted one."""
        import dataclasses

        opt = self.optimizer
        sd = dict(config=dataclasses.asdict(self.cfg), iteration=self.steps_done,
                  params={k: getattr(self.params, k).detach().clone() for k in self._PARAM_NAMES},
                  optimizer=dict(exp_avg=[m.clone() for m in opt.exp_avg], exp_avg_sq=[v.clone() for v in opt.exp_avg_sq],
                                 step=opt.step_count, lr=opt.lr, betas=opt.betas, eps=opt.eps),
                  refine=None, source_generator=None)
        if self.refine_stats is not None:
            sd["refine"] = dict(importance=self.refine_stats.importance.clone(), visits=self.refine_stats.visits.clone(),
                                log=[dict(r) for r in self.refine_log], generator=self.refine_gen.get_state())
        if self.source is not None:
            sd["source_generator"] = self.source["gen"].get_state()
        return sd

    def load_state_dict(self, sd: dict) -> None:
        """Restores a state_dict() into this trainer (same batches / frame source and refinement
        schedule). Parameters of the same size are copied in place (the captured graphs stay
        valid); a different number of Gaussians replaces the buffers and captures again."""
        dev = self.params.means.device
        new = {k: sd["params"][k].to(dev, torch.float32) for k in self._PARAM_NAMES}
        opt = self.optimizer
        same = all(getattr(self.params, k).shape == new[k].shape for k in self._PARAM_NAMES)
        if same:
            for k in self._PARAM_NAMES:
                getattr(self.params, k).copy_(new[k])
            for dst, src in zip(opt.exp_avg + opt.exp_avg_sq, sd["optimizer"]["exp_avg"] + sd["optimizer"]["exp_avg_sq"]):
                dst.copy_(src.to(dev))
        else:
            for k in self._PARAM_NAMES:
                setattr(self.params, k, new[k].contiguous())
            opt.params = self.params.tensors()
            opt.exp_avg = [m.to(dev).contiguous() for m in sd["optimizer"]["exp_avg"]]
            opt.exp_avg_sq = [v.to(dev).contiguous() for v in sd["optimizer"]["exp_avg_sq"]]
        opt.step_count = int(sd["optimizer"]["step"])
        self.steps_done = int(sd["iteration"])
        if sd.get("refine") is not None and self.refine_stats is not None:
            from .refine import RefineStats

            r = sd["refine"]
            if not same:
                self.refine_stats = RefineStats(new["means"].shape[0], dev)
            self.refine_stats.importance.copy_(r["importance"].to(dev))
            self.refine_stats.visits.copy_(r["visits"].to(dev))
            self.refine_log = [dict(x) for x in r["log"]]
            self.refine_gen.set_state(r["generator"])
        if not same:
            self._rebuffer()  # primes the capacity with draws of its own: before the states below
        if sd.get("source_generator") is not None and self.source is not None:
            self.source["gen"].set_state(sd["source_generator"])

    def save(self, path) -> None:
        """torch.save of state_dict() (tensors moved to the host)."""
        def host(x):
            if torch.is_tensor(x):
                return x.cpu()
            if isinstance(x, dict):
                return {k: host(v) for k, v in x.items()}
            if isinstance(x, (list, tuple)):
                return type(x)(host(v) for v in x)
            return x

        torch.save(host(self.state_dict()), path)

    def load(self, path) -> None:
        self.load_state_dict(torch.load(path, map_location="cpu", weights_only=False))

    def losses(self, batch_index: int = 0) -> torch.Tensor:
        return self._batches[batch_index]["stats"].cpu()

    def check(self) -> None:
        if self.source is not None:
            self.source["source"].check()
        for k, bt in enumerate(self._batches):
            if bt["binning"] is None:
                continue
            total, flags = UG.read_status(bt["binning"])
            if flags:
                raise RuntimeError(f"trainer batch {k}: binning flags {flags} ({total} instances, "
                                   f"capacity {bt['capacity']})")
