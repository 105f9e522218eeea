"""Host side of the UltraGauss slice splatting path over the C ABI.

One ``UGBinning`` is the result of binning G Gaussians against one or more probe slices
("frames") in a single launch sequence; forward, backward, the per-pixel candidate lists
and the reference-format sort keys are all read from it. Frames in one binning may have
different sizes (the batched form); the plain drop-in renderer bins one frame per call.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import torch

from . import _lib

TILE = 16


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _set_device(dev: torch.device) -> None:
    _lib.check(_lib.call("us3d_set_device", dev.index if dev.index is not None else torch.cuda.current_device()),
               "us3d_set_device")


@dataclass
class SliceSpec:
    """Geometry of one planar slice (the reference's UltraGaussRenderConfig + SliceGeometry)."""

    height: int
    width: int
    lateral_spacing: float
    axial_spacing: float
    axial_near: float
    lateral_col_offset: float
    origin: torch.Tensor  # (3,)
    axis_lat: torch.Tensor
    axis_ax: torch.Tensor
    axis_ele: torch.Tensor
    # (first Gaussian, count) of the Gaussian set this frame renders; None: all Gaussians.
    # Frames of independent sweeps, each with its own Gaussians, then render in one call over
    # the concatenated parameters.
    gaussian_set: Optional[Tuple[int, int]] = None


@dataclass
class FrameTable:
    table: torch.Tensor  # (F, 24) float32 on device, int fields bit-cast
    n_frames: int
    n_tiles: int
    n_pixels: int
    tile_offsets: List[int]
    tile_counts: List[int]
    pixel_offsets: List[int]
    sizes: List[tuple]
    gaussian_sets: bool = False


def build_frame_table(specs: Sequence[SliceSpec], device: torch.device) -> FrameTable:
    """Packs slice geometry into the device array of ``us3d_slice_frame``."""
    F = len(specs)
    ints = torch.zeros((F, 8), dtype=torch.int32)
    scal = torch.zeros((F, 4), dtype=torch.float32)
    t_off = p_off = 0
    tile_offsets, tile_counts, pixel_offsets, sizes = [], [], [], []
    sets = [getattr(s, "gaussian_set", None) for s in specs]
    use_sets = any(x is not None for x in sets)
    if use_sets:
        if any(x is None for x in sets):
            raise ValueError("either every frame names its Gaussian set or none does")
        prev = None
        for i, (off, cnt) in enumerate(sets):
            if off < 0 or cnt < 0 or off + cnt > 0x7FFFFFFF:
                raise ValueError(f"frame {i}: bad Gaussian set ({off}, {cnt})")
            if prev is not None and (off, cnt) != prev and off < prev[0] + prev[1]:
                raise ValueError(f"frame {i}: Gaussian sets must be contiguous runs in increasing, "
                                 f"non-overlapping order (set ({off}, {cnt}) after {prev})")
            prev = (off, cnt)
    for i, s in enumerate(specs):
        H, W = int(s.height), int(s.width)
        tx, ty = (W + TILE - 1) // TILE, (H + TILE - 1) // TILE
        go, gc = sets[i] if use_sets else (0, 0)
        ints[i, :8] = torch.tensor([H, W, tx, ty, p_off, t_off, go, gc], dtype=torch.int32)
        scal[i] = torch.tensor([s.lateral_spacing, s.axial_spacing, s.axial_near, s.lateral_col_offset],
                               dtype=torch.float32)
        tile_offsets.append(t_off)
        tile_counts.append(tx * ty)
        pixel_offsets.append(p_off)
        sizes.append((H, W))
        t_off += tx * ty
        p_off += H * W
    if F:
        axes = torch.stack(
            [torch.cat([s.origin.reshape(3), s.axis_lat.reshape(3), s.axis_ax.reshape(3), s.axis_ele.reshape(3)])
             for s in specs]
        ).to(device=device, dtype=torch.float32)
        host_tail = torch.cat([scal, ints.view(torch.float32)], dim=1).to(device, non_blocking=False)
        table = torch.cat([axes, host_tail], dim=1).contiguous()
    else:
        table = torch.zeros((0, 24), dtype=torch.float32, device=device)
    return FrameTable(table, F, t_off, p_off, tile_offsets, tile_counts, pixel_offsets, sizes, use_sets)


# Capacity hints per (G, n_tiles): the last instance total seen, so that steady-state calls
# bin once. A miss costs one extra bin (the total is exact even when the capacity is short).
_capacity_hint: dict = {}


@dataclass
class UGBinning:
    workspace: torch.Tensor
    capacity: int
    total: int
    frames: FrameTable
    n_gauss: int
    chi2: float
    beta: float
    sort_by_depth: bool
    slice_cull: bool = False
    pixels: Optional[torch.Tensor] = None
    counts: Optional[torch.Tensor] = None


def _check_params(means, tril, opac, inten):
    G = means.shape[0]
    if means.shape != (G, 3) or tril.shape != (G, 6) or opac.reshape(-1).shape[0] != G or inten.reshape(-1).shape[0] != G:
        raise ValueError(
            f"UltraGauss parameter shapes must be means (G,3), precision_tril (G,6), opacities (G,), "
            f"intensities (G,); got {tuple(means.shape)}, {tuple(tril.shape)}, {tuple(opac.shape)}, {tuple(inten.shape)}"
        )
    return G


def bin_gaussians(means: torch.Tensor, tril: torch.Tensor, opac: torch.Tensor, inten: torch.Tensor,
                  frames: FrameTable, chi2: float, beta: float, sort_by_depth: bool = True,
                  capacity: Optional[int] = None, sync_check: bool = True,
                  slice_cull_pixels: Optional[torch.Tensor] = None, logit_attributes: bool = False) -> UGBinning:
    """Runs the mapper for all frames. With ``sync_check`` the instance total is read back
    (one stream synchronisation) and the binning is redone with a larger capacity if needed.
    Passing the frames' pixel positions as ``slice_cull_pixels`` drops the tiles a Gaussian's
    chi-square ellipse cannot reach (same images and gradients; no per-pixel candidate counts
    or lists afterwards). With ``logit_attributes`` the opacities and intensities are raw
    logits, activated by the logistic function inside the binning (the gradients that
    ``backward`` returns are then still w.r.t. the activated values)."""
    G = _check_params(means, tril, opac, inten)
    dev = means.device
    _set_device(dev)
    cull = slice_cull_pixels is not None
    key = (G, frames.n_tiles, cull)
    cap = int(capacity if capacity is not None else _capacity_hint.get(key, max(4096, 4 * G)))
    for _attempt in range(3):
        nbytes = _lib.call("us3d_ug_workspace_bytes", G, frames.n_frames, frames.n_tiles, frames.n_pixels, cap)
        ws = torch.empty(int(nbytes), dtype=torch.uint8, device=dev)
        st = _lib.call(
            "us3d_ug_bin_ex", _ptr(ws), int(nbytes), _ptr(frames.table), frames.n_frames, frames.n_tiles,
            frames.n_pixels, G, _ptr(means), _ptr(tril), _ptr(opac), _ptr(inten), float(chi2), float(beta),
            int(bool(sort_by_depth)), cap, _ptr(slice_cull_pixels) if cull else None,
            (_lib.UG_BIN_SLICE_CULL if cull else 0) | (_lib.UG_BIN_LOGIT_ATTRIBUTES if logit_attributes else 0)
            | (_lib.UG_BIN_GAUSSIAN_SETS if frames.gaussian_sets else 0), _stream(),
        )
        _lib.check(st, "us3d_ug_bin_ex")
        b = UGBinning(ws, cap, -1, frames, G, float(chi2), float(beta), bool(sort_by_depth), cull)
        if not sync_check:
            return b
        total, flags = read_status(b)
        if flags & 2:
            raise RuntimeError("us3d_ug_bin: inconsistent frame table")
        b.total = total
        if not flags:
            _capacity_hint[key] = max(4096, int(total * 1.25) + 1024)
            return b
        if total > 0x7FFFFFFF:
            raise RuntimeError(f"us3d_ug_bin: {total} instances exceed the int32 index range")
        cap = int(total * 1.25) + 1024
    raise RuntimeError("us3d_ug_bin: capacity retry failed")


def read_status(b: UGBinning):
    total = ctypes.c_int64(0)
    flags = ctypes.c_int32(0)
    _lib.check(_lib.call("us3d_ug_read_status", _ptr(b.workspace), ctypes.byref(total), ctypes.byref(flags),
                         _stream()), "us3d_ug_read_status")
    return int(total.value), int(flags.value)


def forward(b: UGBinning, pixels: torch.Tensor, bg_alpha: float, bg_intensity: float,
            want_counts: bool = True):
    """Returns image, alpha, depth (n_pixels,) and the per-pixel candidate counts (int32)."""
    P = b.frames.n_pixels
    dev = pixels.device
    image = torch.empty(P, dtype=torch.float32, device=dev)
    alpha = torch.empty(P, dtype=torch.float32, device=dev)
    depth = torch.empty(P, dtype=torch.float32, device=dev)
    # a slice-culled binning has no per-pixel candidate counts
    counts = torch.empty(P, dtype=torch.int32, device=dev) if (want_counts and not b.slice_cull) else None
    st = _lib.call(
        "us3d_ug_forward", _ptr(b.workspace), _ptr(b.frames.table), b.frames.n_frames, b.frames.n_tiles, P,
        b.n_gauss, b.capacity, _ptr(pixels), b.chi2, b.beta, float(bg_alpha), float(bg_intensity), _ptr(image),
        _ptr(alpha), _ptr(depth), _ptr(counts), _stream(),
    )
    _lib.check(st, "us3d_ug_forward")
    # No reference to the outputs here: an autograd function keeping the binning on its ctx
    # would otherwise form a cycle (output -> node -> binning -> output) that only the cyclic
    # garbage collector frees, keeping each step's workspace alive for an unknown time.
    b.pixels = pixels
    b.counts = counts
    return image, alpha, depth, counts


# Backward scratch (the per-instance partials) kept per (device, stream): the partials are
# consumed by the same call's reduction, and a later call on the same stream runs after it, so
# every call on a stream can reuse one buffer instead of allocating ~48 bytes per instance.
_SCRATCH = {}


def _backward_scratch(dev: torch.device, nbytes: int) -> torch.Tensor:
    if torch.cuda.is_current_stream_capturing():
        # a graph keeps its own (private pool) buffer: the cached one may be freed later
        return torch.empty(max(nbytes, 16), dtype=torch.uint8, device=dev)
    key = (dev.index if dev.index is not None else torch.cuda.current_device(),
           torch.cuda.current_stream(dev).cuda_stream)
    buf = _SCRATCH.get(key)
    if buf is None or buf.numel() < nbytes:
        _SCRATCH.pop(key, None)
        buf = torch.empty(max(nbytes, 16), dtype=torch.uint8, device=dev)
        _SCRATCH[key] = buf
    return buf


def release_scratch() -> None:
    """Frees the backward scratch buffers kept per stream (they are re-created on demand)."""
    _SCRATCH.clear()


def backward(b: UGBinning, pixels: torch.Tensor, d_image: torch.Tensor, d_alpha: torch.Tensor,
             d_depth: torch.Tensor, saved_alpha: torch.Tensor, bg_alpha: float, bg_intensity: float,
             scratch: Optional[torch.Tensor] = None, out=None):
    """Gradients w.r.t. means (G,3), precision_tril (G,6), opacities (G,), intensities (G,)."""
    G = b.n_gauss
    dev = pixels.device
    sbytes = int(_lib.call("us3d_ug_backward_scratch_bytes", b.capacity))
    if scratch is None or scratch.numel() < sbytes:
        scratch = _backward_scratch(dev, sbytes)
    if out is None:
        out = (
            torch.empty((G, 3), dtype=torch.float32, device=dev),
            torch.empty((G, 6), dtype=torch.float32, device=dev),
            torch.empty((G,), dtype=torch.float32, device=dev),
            torch.empty((G,), dtype=torch.float32, device=dev),
        )
    dm, dt, do, di = out
    st = _lib.call(
        "us3d_ug_backward", _ptr(b.workspace), _ptr(b.frames.table), b.frames.n_frames, b.frames.n_tiles,
        b.frames.n_pixels, G, b.capacity, _ptr(pixels), _ptr(d_image), _ptr(d_alpha), _ptr(d_depth),
        _ptr(saved_alpha), b.chi2, b.beta, float(bg_alpha), float(bg_intensity), _ptr(scratch), int(scratch.numel()),
        _ptr(dm), _ptr(dt), _ptr(do), _ptr(di), _stream(),
    )
    _lib.check(st, "us3d_ug_backward")
    return dm, dt, do, di


def loss(frames: FrameTable, image: torch.Tensor, target: torch.Tensor, l1_weight: float = 1.0,
         ssim_weight: float = 0.0, scratch: Optional[torch.Tensor] = None, out=None):
    """Per-frame loss l1_weight * mean|x - y| + ssim_weight * (1 - global SSIM) of the frames'
    images against their targets. Returns (stats (F,8) float64: mean x, mean y, var x, var y,
    cov xy, mean |x - y|, SSIM, loss; coef (F,4) float32: the per-frame coefficients of the
    loss gradient, consumed by ``backward_loss``). Never synchronises."""
    dev = image.device
    F = frames.n_frames
    sbytes = int(_lib.call("us3d_ug_loss_scratch_bytes", F))
    if scratch is None or scratch.numel() < sbytes:
        scratch = torch.empty(max(sbytes, 16), dtype=torch.uint8, device=dev)
    if out is None:
        out = (torch.empty((F, 8), dtype=torch.float64, device=dev), torch.empty((F, 4), dtype=torch.float32, device=dev))
    stats, coef = out
    _lib.check(_lib.call("us3d_ug_loss", _ptr(frames.table), F, frames.n_pixels, _ptr(image), _ptr(target),
                         float(l1_weight), float(ssim_weight), _ptr(scratch), int(scratch.numel()), _ptr(stats),
                         _ptr(coef), _stream()), "us3d_ug_loss")
    return stats, coef


def backward_loss(b: UGBinning, pixels: torch.Tensor, image: torch.Tensor, target: torch.Tensor,
                  coef: torch.Tensor, saved_alpha: torch.Tensor, bg_alpha: float, bg_intensity: float,
                  scratch: Optional[torch.Tensor] = None, out=None):
    """``backward`` with dL/dimage taken from the fused per-frame loss (``loss``'s coefficients)
    and zero dL/dalpha, dL/ddepth."""
    G = b.n_gauss
    dev = pixels.device
    sbytes = int(_lib.call("us3d_ug_backward_scratch_bytes", b.capacity))
    if scratch is None or scratch.numel() < sbytes:
        scratch = _backward_scratch(dev, sbytes)
    if out is None:
        out = (
            torch.empty((G, 3), dtype=torch.float32, device=dev),
            torch.empty((G, 6), dtype=torch.float32, device=dev),
            torch.empty((G,), dtype=torch.float32, device=dev),
            torch.empty((G,), dtype=torch.float32, device=dev),
        )
    dm, dt, do, di = out
    st = _lib.call(
        "us3d_ug_backward_loss", _ptr(b.workspace), _ptr(b.frames.table), b.frames.n_frames, b.frames.n_tiles,
        b.frames.n_pixels, G, b.capacity, _ptr(pixels), _ptr(image), _ptr(target), _ptr(coef), _ptr(saved_alpha),
        b.chi2, b.beta, float(bg_alpha), float(bg_intensity), _ptr(scratch), int(scratch.numel()), _ptr(dm),
        _ptr(dt), _ptr(do), _ptr(di), _stream(),
    )
    _lib.check(st, "us3d_ug_backward_loss")
    return dm, dt, do, di


def pixel_csr(b: UGBinning, pixels: torch.Tensor, counts: torch.Tensor):
    """The reference's per-pixel candidate CSR: (offsets (P,) int32, indices (K,) int32)."""
    P = b.frames.n_pixels
    dev = pixels.device
    if P == 0:
        return torch.zeros(0, dtype=torch.int32, device=dev), torch.zeros(0, dtype=torch.int32, device=dev)
    c64 = counts.to(torch.int64)
    ends = torch.cumsum(c64, 0)
    offsets = (ends - c64).to(torch.int32)
    total = int(ends[-1].item())
    indices = torch.empty(total, dtype=torch.int32, device=dev)
    if total > 0:
        st = _lib.call(
            "us3d_ug_pixel_csr", _ptr(b.workspace), _ptr(b.frames.table), b.frames.n_frames, b.frames.n_tiles, P,
            b.n_gauss, b.capacity, _ptr(pixels), b.chi2, b.beta, _ptr(offsets), _ptr(indices), _stream(),
        )
        _lib.check(st, "us3d_ug_pixel_csr")
    return offsets, indices


def export_bins(b: UGBinning, frame: int = 0):
    """Sorted keys (int64), values (int32) and tile ranges of one frame, reference format."""
    ft = b.frames
    t_off, nt = ft.tile_offsets[frame], ft.tile_counts[frame]
    first = ctypes.c_int64(0)
    count = ctypes.c_int64(0)
    _lib.check(_lib.call("us3d_ug_frame_instances", _ptr(b.workspace), ft.n_tiles, t_off, nt, ctypes.byref(first),
                         ctypes.byref(count), _stream()), "us3d_ug_frame_instances")
    dev = b.workspace.device
    n = int(count.value)
    keys = torch.empty(n, dtype=torch.int64, device=dev)
    vals = torch.empty(n, dtype=torch.int32, device=dev)
    rs = torch.empty(nt, dtype=torch.int32, device=dev)
    re = torch.empty(nt, dtype=torch.int32, device=dev)
    _lib.check(_lib.call("us3d_ug_export_bins", _ptr(b.workspace), ft.n_tiles, t_off, nt, _ptr(keys), _ptr(vals),
                         _ptr(rs), _ptr(re), _stream()), "us3d_ug_export_bins")
    return keys, vals, rs, re
