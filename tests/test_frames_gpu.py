"""Frame batches assembled on the device (us3d_frames_gather) against the reference dataset's
host-side construction (NpzUltrasoundDataset.get_frame, pipeline_god_file.py:212-306):
generated pixel grids bit-identical to the reference's PyTorch arithmetic, targets with its
8-bit scaling, explicit pixel positions gathered as stored, an NPZ in the reference's layout,
out-of-range indices reported, and the trainer drawing its batches on the device."""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _ref_normalize(x):
    return x / torch.clamp(torch.linalg.norm(x), min=1.0e-8)


def _ref_pixel_positions(h, w, origin, lat, ax, dlat, dax, near, center_lateral, device):
    """The reference's generated grid, restated with the same PyTorch operations."""
    u = torch.arange(w, device=device, dtype=torch.float32)
    v = torch.arange(h, device=device, dtype=torch.float32)
    center = (w - 1) * 0.5 if center_lateral else 0.0
    lateral_mm = (u - center) * float(dlat)
    axial_mm = float(near) + v * float(dax)
    yy, xx = torch.meshgrid(axial_mm, lateral_mm, indexing="ij")
    pix = origin.view(1, 1, 3) + xx[..., None] * lat.view(1, 1, 3) + yy[..., None] * ax.view(1, 1, 3)
    return pix.reshape(-1, 3).contiguous()


def _dataset(n=6, h=37, w=50, u8=True, seed=0):
    rng = np.random.default_rng(seed)
    images = rng.integers(0, 256, (n, h, w), dtype=np.uint8) if u8 else rng.random((n, h, w), dtype=np.float32)
    geo = {k: rng.normal(size=(n, 3)).astype(np.float32) * (20.0 if k == "o" else 1.0) for k in ("o", "l", "a", "e")}
    return images, geo


@pytest.mark.parametrize("center,near", [(True, 0.0), (False, 3.7)])
def test_generated_grid_and_targets_match_reference(center, near, cuda_device):
    from us3d_b200.frames import DeviceFrameSource

    dev = cuda_device
    images, g = _dataset()
    src = DeviceFrameSource(images, g["o"], g["l"], g["a"], g["e"], 0.3, 0.17, near, center, device=dev)
    idx = torch.tensor([4, 0, 4, 2], dtype=torch.int64, device=dev)
    table, pix, tgt = src.batch(idx)
    src.check()
    hw = 37 * 50
    rec = table.table.cpu()
    for f, k in enumerate(idx.tolist()):
        o = torch.from_numpy(g["o"][k]).to(dev)
        lat = _ref_normalize(torch.from_numpy(g["l"][k]).to(dev))
        ax = _ref_normalize(torch.from_numpy(g["a"][k]).to(dev))
        ele = _ref_normalize(torch.from_numpy(g["e"][k]).to(dev))
        ref = _ref_pixel_positions(37, 50, o, lat, ax, 0.3, 0.17, near, center, dev)
        assert torch.equal(pix[f * hw:(f + 1) * hw], ref), f
        want = torch.from_numpy(images[k].astype(np.float32).reshape(-1) / 255.0)
        assert torch.equal(tgt[f * hw:(f + 1) * hw].cpu(), want), f
        assert torch.equal(rec[f, 0:12], torch.cat([o, lat, ax, ele]).cpu())
        ints = rec[f, 16:24].view(torch.int32).tolist()
        assert ints[:6] == [37, 50, 4, 3, f * hw, f * 12]


def test_float_images_scaling_and_explicit_pixels(cuda_device):
    from us3d_b200.frames import DeviceFrameSource

    dev = cuda_device
    images, g = _dataset(u8=False)
    pp = np.random.default_rng(3).normal(size=(6, 37 * 50, 3)).astype(np.float32)
    for scale in (1.0, 200.0):
        src = DeviceFrameSource(images * scale, g["o"], g["l"], g["a"], g["e"], 0.3, 0.17, 0.0, True,
                                pixel_positions=pp, device=dev)
        idx = torch.tensor([1, 5], dtype=torch.int64, device=dev)
        _, pix, tgt = src.batch(idx)
        for f, k in enumerate((1, 5)):
            assert torch.equal(pix[f * 1850:(f + 1) * 1850].cpu(), torch.from_numpy(pp[k]))
            x = (images[k] * scale).astype(np.float32).reshape(-1)
            want = x / 255.0 if scale > 1.5 else x
            assert torch.equal(tgt[f * 1850:(f + 1) * 1850].cpu(), torch.from_numpy(want.astype(np.float32)))


def test_npz_layout_and_out_of_range_index(tmp_path, cuda_device):
    from us3d_b200.frames import DeviceFrameSource

    dev = cuda_device
    images, g = _dataset(n=3, h=20, w=24)
    path = tmp_path / "sweep.npz"
    np.savez(path, images=images[:, None], probe_origin_world=g["o"][:3], axis_lateral_world=g["l"][:3],
             axis_axial_world=g["a"][:3], axis_elevational_world=np.array([0, 0, 1], np.float32))
    src = DeviceFrameSource.from_npz(path, 0.5, 0.5, 1.0, device=dev)
    assert (src.n, src.height, src.width) == (3, 20, 24)
    table, pix, tgt = src.batch(torch.tensor([2], dtype=torch.int64, device=dev))
    src.check()
    ref = _ref_pixel_positions(20, 24, torch.from_numpy(g["o"][2]).to(dev),
                               _ref_normalize(torch.from_numpy(g["l"][2]).to(dev)),
                               _ref_normalize(torch.from_numpy(g["a"][2]).to(dev)), 0.5, 0.5, 1.0, True, dev)
    assert torch.equal(pix, ref)
    src.batch(torch.tensor([0, 3], dtype=torch.int64, device=dev))  # 3 is outside the dataset
    with pytest.raises(IndexError):
        src.check()


def test_trainer_on_device_batches(cuda_device):
    from us3d_b200 import scenes
    from us3d_b200.frames import DeviceFrameSource
    from us3d_b200.train import TrainConfig, UltraGaussParameters, UltraGaussTrainer

    dev = cuda_device
    sweep = scenes.linear_sweep(8, 64, 80, 0.3, seed=2, cube_mm=32.0)
    rng = np.random.default_rng(1)
    images = rng.integers(0, 256, (8, 64, 80), dtype=np.uint8)
    geo = [torch.stack([getattr(s, k) for s in sweep]).numpy() for k in ("origin", "axis_lat", "axis_ax", "axis_ele")]
    sc = scenes.make_scene(15000, seed=2, cube_mm=32.0)
    out = []
    for graph in (False, True):
        src = DeviceFrameSource(images, *geo, 0.3, 0.3, 0.0, True, device=dev)
        params = UltraGaussParameters.from_points(sc.means.to(dev), sc.intensities.to(dev), init_scale_mm=0.8)
        tr = UltraGaussTrainer.from_source(params, src, batch_size=3, cfg=TrainConfig(lr=5e-3), seed=7, graph=graph)
        for _ in range(4):
            tr.step()
        tr.check()
        out.append([t.cpu().numpy() for t in params.tensors()])
    for a, b in zip(*out):
        assert np.array_equal(a, b)
    assert not np.array_equal(out[0][0], sc.means.numpy())


def _ref_rays_and_pose(w, origin, lat, ax, ele, dlat, center_lateral, device):
    """The reference's generated scanlines and world-to-probe pose (pipeline_god_file.py:308-336),
    restated with the same PyTorch operations."""
    u = torch.arange(w, device=device, dtype=torch.float32)
    center = (w - 1) * 0.5 if center_lateral else 0.0
    lateral_mm = (u - center) * float(dlat)
    origins = origin.view(1, 3) + lateral_mm[:, None] * lat.view(1, 3)
    dirs = ax.view(1, 3).expand(w, 3).contiguous()
    r = torch.stack([lat, ax, ele], dim=0)
    t = -r.matmul(origin)
    pose = torch.eye(4, device=device, dtype=torch.float32)
    pose[:3, :3] = r
    pose[:3, 3] = t
    return origins, dirs, pose


@pytest.mark.parametrize("center", [True, False])
def test_generated_rays_and_poses_match_reference(center, cuda_device):
    from us3d_b200.frames import DeviceFrameSource

    dev = cuda_device
    images, g = _dataset()
    src = DeviceFrameSource(images, g["o"], g["l"], g["a"], g["e"], 0.3, 0.17, 0.0, center, device=dev)
    idx = torch.tensor([3, 3, 0, 5, 1], dtype=torch.int64, device=dev)
    origins, dirs, pose = src.geometry(idx)
    src.check()
    for f, k in enumerate(idx.tolist()):
        o = torch.from_numpy(g["o"][k]).to(dev)
        lat, ax, ele = (_ref_normalize(torch.from_numpy(g[c][k]).to(dev)) for c in ("l", "a", "e"))
        ro, rd, rp = _ref_rays_and_pose(50, o, lat, ax, ele, 0.3, center, dev)
        assert torch.equal(origins[f], ro), f
        assert torch.equal(dirs[f], rd), f
        assert torch.equal(pose[f, :3, :3], rp[:3, :3]) and torch.equal(pose[f, 3], rp[3]), f
        # the translation is a 3-term dot product whose summation order the reference leaves to torch
        torch.testing.assert_close(pose[f, :3, 3], rp[:3, 3], rtol=1e-6, atol=1e-5)


def test_stored_rays_and_poses_and_bad_index(cuda_device, tmp_path):
    from us3d_b200.frames import DeviceFrameSource

    dev = cuda_device
    images, g = _dataset(n=4, h=9, w=11)
    rng = np.random.default_rng(3)
    ro = rng.normal(size=(4, 11, 3)).astype(np.float32)
    rd = rng.normal(size=(4, 11, 3)).astype(np.float32)
    pose = rng.normal(size=(4, 4)).astype(np.float32)  # one pose shared by every frame
    path = tmp_path / "frames.npz"
    np.savez(path, images=images, probe_origin_world=g["o"], axis_lateral_world=g["l"], axis_axial_world=g["a"],
             axis_elevational_world=g["e"], ray_origins=ro, ray_dirs=rd, pose_world_to_probe=pose)
    src = DeviceFrameSource.from_npz(path, 0.3, 0.17, device=dev)
    idx = torch.tensor([2, 0, 3], dtype=torch.int64, device=dev)
    origins, dirs, poses = src.geometry(idx)
    src.check()
    for f, k in enumerate(idx.tolist()):
        assert torch.equal(origins[f].cpu(), torch.from_numpy(ro[k]))
        assert torch.equal(dirs[f].cpu(), torch.from_numpy(rd[k]))
        assert torch.equal(poses[f].cpu(), torch.from_numpy(pose))
    src.geometry(torch.tensor([1, 7], dtype=torch.int64, device=dev))
    with pytest.raises(IndexError):
        src.check()


def test_camera_fields_on_device(cuda_device):
    """The UltraGS camera fields gathered on the GPU for a device index tensor equal the stored
    per-frame values (shared / absent ones broadcast as the reference's loader does)."""
    from us3d_b200.frames import DeviceFrameSource

    images, g = _dataset(n=3, h=20, w=24)
    rng = np.random.default_rng(5)
    view = rng.normal(size=(3, 4, 4)).astype(np.float32)
    proj = rng.normal(size=(4, 4)).astype(np.float32)
    src = DeviceFrameSource(images, g["o"][:3], g["l"][:3], g["a"][:3], np.array([0, 0, 1], np.float32), 0.5, 0.5,
                            device=cuda_device, viewmatrix=view, projmatrix=proj, tanfovx=np.float32(0.25))
    idx = torch.tensor([2, 0], dtype=torch.int64, device=cuda_device)
    v, p, c, tx, ty = src.camera(idx)
    src.check()
    assert torch.equal(v.cpu(), torch.from_numpy(view[[2, 0]]))
    assert torch.equal(p.cpu(), torch.from_numpy(np.stack([proj, proj])))
    assert torch.equal(c.cpu(), torch.from_numpy(g["o"][[2, 0]].astype(np.float32)))
    assert torch.equal(tx.cpu(), torch.tensor([0.25, 0.25])) and torch.equal(ty.cpu(), torch.tensor([0.5, 0.5]))
