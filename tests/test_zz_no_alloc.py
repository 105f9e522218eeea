"""The UltraGauss render entry point that allocates no device memory.

It serves callers that cannot call cudaMalloc (an application that owns the device memory
pool, or a real-time pipeline that must not allocate or stall while it runs): its scratch
is a fixed file-scope device array inside libus3d_b200.so. Called through the C ABI, it
must give the same image, alpha, depth and candidate counts as the regular
us3d_ug_bin + us3d_ug_forward path, on two calls in a row (the array keeps the previous
call's contents, so the second call shows nothing stale leaks through), and must reject
sizes whose workspace does not fit the array.

This file is named to be collected last, so a run that stops at the first failure has
already run every other test.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from ug_helpers import rel_l2

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-5


def _inputs(device, G, H, W, spacing, seed, log_scale_mean=0.0, in_plane=False):
    from us3d_b200 import scenes
    from us3d_b200 import ultragauss as UG

    sc = scenes.make_scene(G, seed=seed, log_scale_mean=log_scale_mean)
    fr = scenes.linear_sweep(4, H, W, spacing, seed=seed)[1]
    if in_plane:  # every mean moved onto the frame's plane: no Gaussian is culled
        ele = (sc.means - fr.origin) @ fr.axis_ele
        sc.means = (sc.means - ele[:, None] * fr.axis_ele[None, :]).contiguous()
    sc = sc.to(device)
    spec = UG.SliceSpec(H, W, spacing, spacing, 0.0, fr.lateral_col_offset, fr.origin, fr.axis_lat, fr.axis_ax,
                        fr.axis_ele)
    frames = UG.build_frame_table([spec], device)
    return sc, frames, fr.pixels.to(device)


def _noalloc(sc, frames, pixels, sort=True, bg_a=1e-6, bg_i=0.0):
    from us3d_b200 import _lib

    L = _lib.load()
    P = frames.n_pixels
    dev = pixels.device
    img = torch.full((P,), float("nan"), device=dev)
    alpha = torch.full((P,), float("nan"), device=dev)
    depth = torch.full((P,), float("nan"), device=dev)
    counts = torch.full((P,), -1, dtype=torch.int32, device=dev)
    n_inst = ctypes.c_int64(-1)
    st = L.us3d_ug_render_noalloc(
        frames.table.data_ptr(), frames.n_frames, frames.n_tiles, P, sc.means.shape[0], sc.means.data_ptr(),
        sc.precision_tril.contiguous().data_ptr(), sc.opacities.data_ptr(), sc.intensities.data_ptr(),
        pixels.data_ptr(), 7.815, 1e-4, int(sort), bg_a, bg_i, img.data_ptr(), alpha.data_ptr(), depth.data_ptr(),
        counts.data_ptr(), ctypes.byref(n_inst), torch.cuda.current_stream().cuda_stream)
    return st, img, alpha, depth, counts, int(n_inst.value)


@pytest.mark.parametrize("G,H,W,spacing,seed,sort", [(20000, 256, 256, 0.25, 0, True), (6000, 100, 180, 0.4, 1, False)])
def test_noalloc_matches_regular_path(G, H, W, spacing, seed, sort, cuda_device):
    from us3d_b200 import _lib
    from us3d_b200 import ultragauss as UG

    sc, frames, pixels = _inputs(cuda_device, G, H, W, spacing, seed)
    b = UG.bin_gaussians(sc.means, sc.precision_tril.contiguous(), sc.opacities, sc.intensities, frames, 7.815, 1e-4,
                         sort)
    ref_img, ref_alpha, ref_depth, ref_counts = UG.forward(b, pixels, 1e-6, 0.0)
    torch.cuda.synchronize()
    for call in range(2):  # two calls in a row on the shared array
        st, img, alpha, depth, counts, n_inst = _noalloc(sc, frames, pixels, sort)
        _lib.check(st, "us3d_ug_render_noalloc")
        torch.cuda.synchronize()
        assert n_inst == b.total, (call, n_inst, b.total)
        assert torch.equal(counts, ref_counts), call
        for got, ref in ((img, ref_img), (alpha, ref_alpha), (depth, ref_depth)):
            assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) <= IMG_TOL, call


def test_noalloc_rejects_oversized_inputs(cuda_device):
    from us3d_b200 import _lib

    sc, frames, pixels = _inputs(cuda_device, 800_000, 64, 64, 1.0, 2)  # 800k Gaussians: workspace > 32 MiB
    st, img, *_ = _noalloc(sc, frames, pixels)
    assert st == _lib.US3D_INVALID_ARG
    msg = _lib.load().us3d_last_error().decode()
    assert "exceed the no-allocation scratch" in msg, msg
    torch.cuda.synchronize()
    assert torch.isnan(img).all()  # nothing was launched


def _regular(sc, frames, pixels, sort=True):
    from us3d_b200 import ultragauss as UG

    b = UG.bin_gaussians(sc.means, sc.precision_tril.contiguous(), sc.opacities, sc.intensities, frames, 7.815, 1e-4,
                         sort)
    return b, UG.forward(b, pixels, 1e-6, 0.0)


def test_noalloc_instance_overflow_leaves_outputs(cuda_device):
    from us3d_b200 import _lib

    # 8000 Gaussians of about 12 mm across a 64 mm frame: millions of instances, far more
    # than the scratch holds, while the sizes themselves fit
    sc, frames, pixels = _inputs(cuda_device, 8000, 512, 512, 0.125, 3, log_scale_mean=float(np.log(12.0)))
    b, _ = _regular(sc, frames, pixels)
    torch.cuda.synchronize()
    for call in range(2):
        st, img, alpha, depth, counts, n_inst = _noalloc(sc, frames, pixels)
        assert st == _lib.US3D_CAPACITY_OVERFLOW, (call, st)
        msg = _lib.load().us3d_last_error().decode()
        assert "instances exceed" in msg, msg
        assert n_inst == b.total, (call, n_inst, b.total)
        torch.cuda.synchronize()
        assert torch.isnan(img).all() and torch.isnan(alpha).all() and torch.isnan(depth).all()
        assert (counts == -1).all()


def test_noalloc_single_tile_gaussians(cuda_device):
    from us3d_b200 import _lib

    # 200k Gaussians of about 0.05 mm on the frame's plane: each reaches one or two 16x16
    # tiles, so the surviving (Gaussian, frame) pairs are most of the instances
    sc, frames, pixels = _inputs(cuda_device, 200_000, 512, 512, 0.125, 4, log_scale_mean=float(np.log(0.05)),
                                 in_plane=True)
    b, (ref_img, ref_alpha, ref_depth, ref_counts) = _regular(sc, frames, pixels)
    torch.cuda.synchronize()
    assert b.total < 2 * 200_000, b.total
    for call in range(2):
        st, img, alpha, depth, counts, n_inst = _noalloc(sc, frames, pixels)
        _lib.check(st, "us3d_ug_render_noalloc")
        torch.cuda.synchronize()
        assert n_inst == b.total, (call, n_inst, b.total)
        assert torch.equal(counts, ref_counts), call
        for got, ref in ((img, ref_img), (alpha, ref_alpha), (depth, ref_depth)):
            assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) <= IMG_TOL, call
