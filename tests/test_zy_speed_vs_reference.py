"""Throughput of the reference's own UltraGauss CUDA (built for sm_100a by oracle/build_ref.py)
next to this library on the same B200, the same scene and the same frames: per-frame forward
+ backward with an L1 loss gradient, as the reference's training loop runs it.

Default sizes keep the test short; US3D_SPEED_GAUSSIANS / US3D_SPEED_SIZE / US3D_SPEED_FRAMES
select others (the headline workload is 1000000 / 512 / 16). The measured numbers are printed
(run pytest with -s to see them) and the test asserts that the library's per-frame path is
faster than the reference's."""

from __future__ import annotations

import os
import sys
from pathlib import Path

import pytest
import torch

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def _ref():
    p = ROOT / "oracle" / "_ref"
    if not any(p.glob("ultragauss_ref_C*.so")):
        pytest.skip("reference build not present")
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))
    import ultragauss_ref_C as REF

    return REF


def _time(fn, reps, dev):
    fn()
    torch.cuda.synchronize(dev)
    st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st.record()
    for _ in range(reps):
        fn()
    en.record()
    torch.cuda.synchronize(dev)
    return st.elapsed_time(en) / reps


def test_speed_vs_reference_cuda(cuda_device):
    REF = _ref()
    from us3d_b200 import scenes
    from us3d_b200 import ultragauss as UG

    dev = cuda_device
    G = int(os.environ.get("US3D_SPEED_GAUSSIANS", "200000"))
    S = int(os.environ.get("US3D_SPEED_SIZE", "256"))
    F = int(os.environ.get("US3D_SPEED_FRAMES", "4"))
    spacing = 64.0 / S
    sc = scenes.make_scene(G, seed=0).to(dev)
    sweep = scenes.linear_sweep(F, S, S, spacing, seed=0, step_mm=64.0 / F)
    specs = [UG.SliceSpec(f.height, f.width, f.lateral_spacing, f.axial_spacing, f.axial_near, f.lateral_col_offset,
                          f.origin, f.axis_lat, f.axis_ax, f.axis_ele) for f in sweep]
    pix = [f.pixels.to(dev).contiguous() for f in sweep]
    tgt = torch.rand((F, S * S), generator=torch.Generator().manual_seed(1)).to(dev)
    means, tril = sc.means.contiguous(), sc.precision_tril.contiguous()
    opac, inten = sc.opacities.contiguous(), sc.intensities.contiguous()
    chi2, beta, bga = 7.815, 1e-4, 1e-6

    # reference: MapperForwardCUDA -> ShaderForwardCUDA -> ShaderBackwardCUDA per frame
    mp = torch.nn.functional.pad(means, (0, 1)).contiguous()
    attr = torch.stack([opac, inten], 1).contiguous()
    pp = [torch.nn.functional.pad(p, (0, 1)).contiguous() for p in pix]

    def ref_frame(k):
        f = sweep[k]
        o, l, a, e = (x.to(dev).contiguous() for x in (f.origin, f.axis_lat, f.axis_ax, f.axis_ele))
        counts, offsets, indices = REF.MapperForwardCUDA(pp[k], mp, tril, o, l, a, e, S, S, spacing, spacing,
                                                         f.axial_near, f.lateral_col_offset, chi2, True, beta)
        image, alpha, depth, sic = REF.ShaderForwardCUDA(attr, mp, tril, pp[k], o, e, offsets, counts, indices, bga,
                                                         0.0, chi2, beta)
        dI = torch.sign(image - tgt[k]) / image.numel()
        z = torch.zeros_like(image)
        REF.ShaderBackwardCUDA(dI, z, z, attr, mp, tril, pp[k], o, e, offsets, counts, indices, sic, alpha, bga, 0.0,
                               chi2, beta)

    tables = [UG.build_frame_table([sp], dev) for sp in specs]

    def ours_frame(k):
        b = UG.bin_gaussians(means, tril, opac, inten, tables[k], chi2, beta, True)
        image, alpha, depth, counts = UG.forward(b, pix[k], bga, 0.0)
        dI = torch.sign(image - tgt[k]) / image.numel()
        z = torch.zeros_like(image)
        UG.backward(b, pix[k], dI, z, z, alpha, bga, 0.0)

    batch_table = UG.build_frame_table(specs, dev)
    allpix = torch.cat(pix)
    alltgt = tgt.reshape(-1)

    def ours_batched():
        b = UG.bin_gaussians(means, tril, opac, inten, batch_table, chi2, beta, True, slice_cull_pixels=allpix)
        image, alpha, depth, _ = UG.forward(b, allpix, bga, 0.0, want_counts=False)
        dI = torch.sign(image - alltgt) / (S * S)
        z = torch.zeros_like(image)
        UG.backward(b, allpix, dI, z, z, alpha, bga, 0.0)

    ms_ref = _time(lambda: [ref_frame(k) for k in range(F)], 1, dev) / F
    ms_ours = _time(lambda: [ours_frame(k) for k in range(F)], 2, dev) / F
    ms_batch = _time(ours_batched, 2, dev) / F
    print(f"\n[speed] {G} Gaussians, {F} frames of {S}x{S} @ {spacing:.4f} mm, fwd+bwd per frame:"
          f"\n[speed] reference CUDA (sm_100a build)  {ms_ref:9.3f} ms/frame  {1000 / ms_ref:9.1f} frames/s"
          f"\n[speed] this library, per frame       {ms_ours:9.3f} ms/frame  {1000 / ms_ours:9.1f} frames/s"
          f"\n[speed] this library, batched + cull  {ms_batch:9.3f} ms/frame  {1000 / ms_batch:9.1f} frames/s"
          f"\n[speed] speed-up per frame {ms_ref / ms_ours:.1f}x, batched {ms_ref / ms_batch:.1f}x")
    assert ms_ours < ms_ref
