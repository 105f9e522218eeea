"""Independent sweeps with their own Gaussian sets in one launch sequence
(US3D_UG_BIN_GAUSSIAN_SETS): frames of three sweeps (different Gaussian counts and frame
sizes) binned, shaded and differentiated together over the concatenated parameters give the
same images and gradients, bit for bit, as each sweep rendered on its own: a frame's tile lists
hold its own set's Gaussians in the same relative order, and each Gaussian's gradient sums its
own instances in the same order."""

from __future__ import annotations

import pytest
import torch

pytestmark = pytest.mark.gpu

SWEEPS = [(3000, 64, 64, 2, 1.0), (12000, 80, 96, 3, 0.7), (700, 128, 128, 2, 0.5)]


def _sweeps():
    from us3d_b200 import scenes
    from us3d_b200 import ultragauss as UG

    out, off = [], 0
    for k, (G, H, W, F, sp) in enumerate(SWEEPS):
        sc = scenes.make_scene(G, seed=40 + k, cube_mm=min(H, W) * sp)
        sw = scenes.linear_sweep(F, H, W, sp, seed=40 + k, cube_mm=min(H, W) * sp)
        specs = [UG.SliceSpec(f.height, f.width, f.lateral_spacing, f.axial_spacing, f.axial_near,
                              f.lateral_col_offset, f.origin, f.axis_lat, f.axis_ax, f.axis_ele) for f in sw]
        out.append((sc, specs, torch.cat([f.pixels for f in sw]), off, G))
        off += G
    return out


@pytest.mark.parametrize("cull", [False, True])
def test_gaussian_sets_match_separate_renders(cull, cuda_device):
    import dataclasses

    from us3d_b200 import ultragauss as UG

    dev = cuda_device
    sw = _sweeps()
    params = [torch.cat([getattr(s[0], k) for s in sw]).to(dev).contiguous()
              for k in ("means", "precision_tril", "opacities", "intensities")]
    specs = [dataclasses.replace(sp, gaussian_set=(off, G)) for sc, ss, px, off, G in sw for sp in ss]
    pixels = torch.cat([s[2] for s in sw]).to(dev).contiguous()
    g = torch.Generator().manual_seed(3)
    d_image = torch.randn(pixels.shape[0], generator=g).to(dev)
    ft = UG.build_frame_table(specs, dev)
    assert ft.gaussian_sets
    b = UG.bin_gaussians(*params, ft, 7.815, 1e-4, True, slice_cull_pixels=pixels if cull else None)
    img, alpha, depth, _ = UG.forward(b, pixels, 1e-6, 0.0, want_counts=False)
    z = torch.zeros_like(img)
    grads = UG.backward(b, pixels, d_image, z, z, alpha, 1e-6, 0.0)
    p0 = 0
    total = 0
    for sc, ss, px, off, G in sw:
        ps = [x[off:off + G].contiguous() for x in params]
        fts = UG.build_frame_table(ss, dev)
        P = px.shape[0]
        pxd = px.to(dev)
        bs = UG.bin_gaussians(*ps, fts, 7.815, 1e-4, True, slice_cull_pixels=pxd if cull else None)
        i2, a2, d2, _ = UG.forward(bs, pxd, 1e-6, 0.0, want_counts=False)
        z2 = torch.zeros_like(i2)
        g2 = UG.backward(bs, pxd, d_image[p0:p0 + P].contiguous(), z2, z2, a2, 1e-6, 0.0)
        for got, ref in ((img, i2), (alpha, a2), (depth, d2)):
            assert torch.equal(got[p0:p0 + P], ref)
        for got, ref in zip(grads, g2):
            assert torch.equal(got[off:off + G], ref)
        total += bs.total
        p0 += P
    assert b.total == total
