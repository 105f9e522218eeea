"""Host-side logic that needs no GPU: lazy intermediates, frame tables, scenes, config
validation, loud failure without CUDA, frame sharding."""

from __future__ import annotations

import numpy as np
import pytest
import torch


def test_lazy_dict_resolves_once_and_only_on_access():
    from us3d_b200.lazy import LazyDict

    calls = []
    d = LazyDict({"b": lambda: calls.append("b") or 2}, a=1)
    assert "b" in d and len(d) == 2 and sorted(d.keys()) == ["a", "b"]
    assert calls == []
    assert d["b"] == 2 and d["b"] == 2 and calls == ["b"]
    d["c"] = 3
    assert dict(d.items()) == {"a": 1, "b": 2, "c": 3}
    e = LazyDict({"x": lambda: 5})
    assert {**e} == {"x": 5} and e.get("x") == 5 and e.pop("x") == 5 and "x" not in e


def test_frame_table_layout():
    from us3d_b200 import scenes
    from us3d_b200 import ultragauss as UG

    frs = [scenes.linear_sweep(3, h, w, 0.5)[i] for i, (h, w) in enumerate([(16, 16), (40, 70), (7, 33)])]
    specs = [UG.SliceSpec(f.height, f.width, 0.5, 0.5, 0.0, f.lateral_col_offset, f.origin, f.axis_lat, f.axis_ax,
                          f.axis_ele) for f in frs]
    ft = UG.build_frame_table(specs, torch.device("cpu"))
    assert ft.table.shape == (3, 24) and ft.table.dtype == torch.float32
    ints = ft.table[:, 16:].contiguous().view(torch.int32)
    assert ints[:, 0].tolist() == [16, 40, 7] and ints[:, 1].tolist() == [16, 70, 33]
    assert ints[:, 2].tolist() == [1, 5, 3] and ints[:, 3].tolist() == [1, 3, 1]
    assert ints[:, 4].tolist() == [0, 256, 256 + 2800] and ints[:, 5].tolist() == [0, 1, 16]
    assert ft.n_tiles == 19 and ft.n_pixels == 256 + 2800 + 231
    assert torch.allclose(ft.table[1, 3:6], frs[1].axis_lat)


def test_scene_is_seeded_and_precision_matches_scales():
    from us3d_b200 import scenes

    a = scenes.make_scene(500, seed=7)
    b = scenes.make_scene(500, seed=7)
    assert torch.equal(a.means, b.means) and torch.equal(a.precision_tril, b.precision_tril)
    t = a.precision_tril.double()
    L = torch.zeros(500, 3, 3, dtype=torch.float64)
    L[:, 0, 0] = t[:, 0] ** 2 + 1e-4
    L[:, 1, 0], L[:, 2, 0] = t[:, 1], t[:, 2]
    L[:, 1, 1] = t[:, 3] ** 2 + 1e-4
    L[:, 2, 1] = t[:, 4]
    L[:, 2, 2] = t[:, 5] ** 2 + 1e-4
    R = scenes.quat_to_rot(a.quats.double())
    lam = R @ torch.diag_embed(1 / a.scales.double() ** 2) @ R.transpose(1, 2)
    assert torch.allclose(L @ L.transpose(1, 2), lam, rtol=1e-5, atol=1e-6)


def test_config_validation_messages():
    from ultragauss_renderer import UltraGaussRenderConfig

    with pytest.raises(ValueError, match="H/W must be positive"):
        UltraGaussRenderConfig(H=0, W=4, lateral_spacing_mm_per_pix=1, axial_spacing_mm_per_pix=1, axial_near_mm=0)
    with pytest.raises(ValueError, match="chi2_threshold must be > 0"):
        UltraGaussRenderConfig(H=4, W=4, lateral_spacing_mm_per_pix=1, axial_spacing_mm_per_pix=1, axial_near_mm=0,
                               chi2_threshold=0)
    c = UltraGaussRenderConfig(H=4, W=9, lateral_spacing_mm_per_pix=1, axial_spacing_mm_per_pix=1, axial_near_mm=0)
    assert c.lateral_col_offset == 4.0


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU behaviour")
def test_renderer_fails_loudly_without_cuda():
    from ultragauss_renderer import SliceGeometry, UltraGaussRenderConfig, UltraGaussRenderer

    cfg = UltraGaussRenderConfig(H=4, W=4, lateral_spacing_mm_per_pix=1, axial_spacing_mm_per_pix=1, axial_near_mm=0)
    g = SliceGeometry(torch.zeros(3), torch.tensor([1.0, 0, 0]), torch.tensor([0, 1.0, 0]), torch.tensor([0, 0, 1.0]))
    with pytest.raises(RuntimeError, match="requires CUDA"):
        UltraGaussRenderer(cfg)(torch.zeros(1, 3), torch.ones(1, 6), torch.ones(1), torch.ones(1), torch.zeros(16, 3), g)


def test_shard_frames_partition():
    from us3d_b200.dist import shard_frames

    for n in (0, 1, 7, 16, 33):
        for w in (1, 2, 3, 8):
            parts = [shard_frames(n, r, w) for r in range(w)]
            assert sum(parts, []) == list(range(n))
            assert max(map(len, parts)) - min(map(len, parts)) <= 1
    with pytest.raises(ValueError):
        shard_frames(4, 2, 2)


def test_device_frame_source_records_on_host():
    """The frame records a DeviceFrameSource keeps (built without a GPU on the CPU device):
    the reference's axis normalisation, spacings, lateral centring and the frame size in the
    us3d_slice_frame layout; 8-bit images scaled by 1/255 when their maximum exceeds 1.5."""
    import numpy as np
    import torch

    from us3d_b200 import _lib
    from us3d_b200.frames import DeviceFrameSource

    rng = np.random.default_rng(0)
    images = rng.integers(0, 256, (4, 10, 12), dtype=np.uint8)
    lat = rng.normal(size=(4, 3)).astype(np.float32)
    src = DeviceFrameSource(images, np.zeros(3, np.float32), lat, [0, 2, 0], None, 0.25, 0.5, 1.5, True,
                            device=torch.device("cpu"))
    assert src.image_format == _lib.IMAGES_U8_DIV255
    rec = src.records
    assert rec.shape == (4, 24)
    ref_lat = torch.from_numpy(lat) / torch.linalg.norm(torch.from_numpy(lat), dim=1, keepdim=True).clamp(min=1e-8)
    assert torch.allclose(rec[:, 3:6], ref_lat, rtol=0, atol=1e-7)
    assert torch.equal(rec[:, 6:9], torch.tensor([[0.0, 1.0, 0.0]]).expand(4, 3))
    assert torch.equal(rec[:, 9:12], torch.tensor([[0.0, 0.0, 1.0]]).expand(4, 3))
    assert torch.equal(rec[0, 12:16], torch.tensor([0.25, 0.5, 1.5, 5.5]))
    assert rec[0, 16:18].view(torch.int32).tolist() == [10, 12]
    flat = DeviceFrameSource(images.astype(np.float32) / 255.0, None, None, None, None, 1.0, 1.0,
                             device=torch.device("cpu"))
    assert flat.image_format == _lib.IMAGES_F32


def test_frame_table_gaussian_sets_validation():
    import dataclasses

    import pytest
    import torch

    from us3d_b200 import scenes
    from us3d_b200 import ultragauss as UG

    fr = scenes.linear_sweep(4, 16, 16, 1.0, seed=0, cube_mm=16.0)
    base = [UG.SliceSpec(f.height, f.width, f.lateral_spacing, f.axial_spacing, f.axial_near, f.lateral_col_offset,
                         f.origin, f.axis_lat, f.axis_ax, f.axis_ele) for f in fr]
    cpu = torch.device("cpu")
    sets = [(0, 10), (0, 10), (10, 5), (20, 1)]
    t = UG.build_frame_table([dataclasses.replace(s, gaussian_set=x) for s, x in zip(base, sets)], cpu)
    assert t.gaussian_sets
    ints = t.table[:, 16:24].contiguous().view(torch.int32)
    assert ints[:, 6].tolist() == [0, 0, 10, 20] and ints[:, 7].tolist() == [10, 10, 5, 1]
    assert not UG.build_frame_table(base, cpu).gaussian_sets
    bad = [
        [(0, 10), (5, 10), (20, 1), (30, 1)],   # overlapping sets
        [(0, 10), (10, 5), (0, 10), (30, 1)],   # a set's frames not contiguous
        [(0, 10), None, (10, 5), (20, 1)],      # some frames without a set
    ]
    for sets in bad:
        with pytest.raises(ValueError):
            UG.build_frame_table([dataclasses.replace(s, gaussian_set=x) for s, x in zip(base, sets)], cpu)


def test_ultragray_profile_schedule_and_ray_stats(monkeypatch):
    """The UltraGray profiling hook's schedule (every n-th call after the warm-up) and its
    per-ray statistics (quantiles over rays with hits, linear interpolation)."""
    import numpy as np
    import torch

    from ultragray_renderer import autograd as A

    monkeypatch.setenv("ULTRAGRAY_PROFILE_EVERY", "3")
    monkeypatch.setenv("ULTRAGRAY_PROFILE_WARMUP", "4")
    assert [s for s in range(1, 16) if A._should_profile(s)] == [6, 9, 12, 15]
    monkeypatch.setenv("ULTRAGRAY_PROFILE_EVERY", "x")
    assert not any(A._should_profile(s) for s in range(1, 16))
    counts = torch.tensor([0, 3, 7, 0, 1, 12, 5], dtype=torch.int32)
    s = A.ray_stats(counts, 28)
    act = np.array([3, 7, 1, 12, 5], np.float64)
    p50, p90, p99 = np.quantile(act, [0.5, 0.9, 0.99])
    assert s == (f"total_hits=28 active_rays=5/7 hits_mean_all={28 / 7:.1f} hits_mean_active={act.mean():.1f} "
                 f"hits_p50={p50:.1f} hits_p90={p90:.1f} hits_p99={p99:.1f} hits_max=12")
    assert "active_rays=0/3" in A.ray_stats(torch.zeros(3, dtype=torch.int32), 0)


def test_workload_time_to_accuracy():
    """Time to reach a held-out L1 target from an evaluation curve of (seconds, frames, L1):
    linear between evaluations, None when never reached."""
    from us3d_b200 import workloads as WL

    c = [(0.0, 0, 0.5), (1.0, 10, 0.3), (2.0, 20, 0.1)]
    assert WL._seconds_to(c, 0.2) == 1.5
    assert WL._seconds_to(c, 0.3) == 1.0
    assert WL._seconds_to(c, 0.05) is None
    assert WL._seconds_to([(0.0, 0, 0.5), (1.0, 8, 0.6), (2.0, 16, 0.4)], 0.45) == 1.75


def _ref_camera(raw, n, idx, origin):
    """The reference loader's UltraGS camera fields for frame idx (pipeline_god_file.py:236-241,
    269-290), restated: stored per-frame or shared values, else identity / probe origin / 0.5."""
    import numpy as np

    def mat(name):
        if name not in raw:
            return np.eye(4, dtype=np.float32)
        a = raw[name].astype(np.float32)
        return a[idx] if a.ndim == 3 and a.shape[0] == n else a

    def arr(name, default):
        if name not in raw:
            return default.astype(np.float32)
        a = raw[name].astype(np.float32)
        return a[idx] if a.ndim >= 2 and a.shape[0] == n else a

    def sca(name, default):
        if name not in raw:
            return np.float32(default)
        a = raw[name].astype(np.float32)
        return np.float32(a[idx] if a.ndim > 0 and a.shape[0] == n else a)

    return mat("viewmatrix"), mat("projmatrix"), arr("camera_center", origin[idx]), sca("tanfovx", 0.5), \
        sca("tanfovy", 0.5)


def test_frame_source_camera_fields(tmp_path):
    """UltraGS camera fields gathered per batch (device gathers; here on the CPU): per-frame,
    shared and absent entries of the reference's NPZ layout, against the reference loader's
    rules; an index outside the dataset is clamped and reported by check()."""
    import numpy as np
    import pytest
    import torch

    from us3d_b200.frames import DeviceFrameSource

    n, h, w = 4, 8, 6
    rng = np.random.default_rng(0)
    base = dict(images=rng.integers(0, 255, (n, h, w), dtype=np.uint8),
                probe_origin_world=rng.normal(size=(n, 3)).astype(np.float32),
                axis_lateral_world=np.array([1, 0, 0], np.float32), axis_axial_world=np.array([0, 1, 0], np.float32),
                axis_elevational_world=np.array([0, 0, 1], np.float32))
    variants = [
        {},
        dict(viewmatrix=rng.normal(size=(n, 4, 4)).astype(np.float32), projmatrix=rng.normal(size=(4, 4)).astype(np.float32),
             camera_center=rng.normal(size=(n, 3)).astype(np.float32), tanfovx=rng.uniform(0.1, 1, n).astype(np.float32),
             tanfovy=np.float32(0.3)),
        dict(camera_center=np.array([1.0, 2.0, 3.0], np.float32), tanfovx=np.float32(0.7)),
    ]
    for k, extra in enumerate(variants):
        raw = dict(base, **extra)
        path = tmp_path / f"c{k}.npz"
        np.savez(path, **raw)
        src = DeviceFrameSource.from_npz(path, 0.5, 0.5, device=torch.device("cpu"))
        idx = torch.tensor([3, 0, 2], dtype=torch.int64)
        got = src.camera(idx)
        for j, i in enumerate(idx.tolist()):
            want = _ref_camera(raw, n, i, base["probe_origin_world"])
            for gv, wv in zip(got, want):
                assert np.array_equal(gv[j].numpy(), np.asarray(wv, np.float32)), (k, i)
        src.check()
        src.camera(torch.tensor([1, 4], dtype=torch.int64))
        with pytest.raises(IndexError):
            src.check()


def test_float_outputs_one_allocation():
    """Gradient outputs carved from one buffer: shapes as asked, each view 16-byte aligned and
    disjoint from the others, the listed ones zero-filled."""
    from us3d_b200._alloc import float_outputs

    shapes = [(5, 3), (5, 1), (5, 0, 3), (4, 4), (7,)]
    out = float_outputs(torch.device("cpu"), shapes, zero=(3,))
    assert [tuple(t.shape) for t in out] == shapes
    assert all(t.dtype == torch.float32 and t.is_contiguous() for t in out)
    assert all(t.data_ptr() % 16 == 0 for t in out if t.numel())
    assert torch.equal(out[3], torch.zeros(4, 4))
    for i, t in enumerate(out):
        t.fill_(float(i + 1))
    for i, t in enumerate(out):
        assert bool((t == float(i + 1)).all())
