"""Reduced versions of the two workloads of us3d_b200.workloads, run end to end on the GPU:
independent sweeps with their own Gaussian sets batched into one graph-replayed step, and
the training workload (layered point cloud, crossing sweeps, speckled targets from a ground
truth, densification / pruning) against the one-frame-per-step form."""

from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


def test_sweeps_workload_small(cuda_device):
    from us3d_b200 import workloads as WL

    b = WL.make_sweep_batch(n_sweeps=4, g_min=2000, g_max=20000, sizes=(64, 96), frames_min=2, frames_max=4,
                            device=cuda_device)
    assert len({s.first_gaussian for s in b.sweeps}) == 4
    out = WL.run_sweeps(b, steps=2, warmup=1)
    assert out["frames"] == sum(s.n_frames for s in b.sweeps)
    assert out["batched"]["instances"] > 0 and out["batched"]["frames_per_s"] > 0
    assert out["plain"]["frames_per_s"] > 0


def test_training_workload_small(cuda_device):
    from us3d_b200 import workloads as WL

    out = WL.run_training(n_init=20_000, n_gt=40_000, n_frames=48, size=128, spacing_mm=0.5, batch=8, steps=100,
                          refine_every=20, plain_frames=64, max_gaussians=40_000, evals=4, device=cuda_device)
    for name in ("batched", "batched_lr_sqrt_batch"):
        b = out[name]
        assert b["frames"] == 800 and b["frames_per_s"] > 0
        assert [r["step"] for r in b["refinements"]] == [20, 40, 60]  # the first 60 % of the steps
        assert sum(r["cloned"] + r["split"] for r in b["refinements"]) > 0  # the top 1 % is densified
        assert len(b["curve"]) == 5 and b["curve"][-1][1] == 800
        assert b["held_out_l1"] < out["held_out_l1_at_start"], out
    assert 0.0 < out["plain"]["held_out_l1"] < 1.0
    assert out["matched_accuracy"]["target_held_out_l1"] == out["plain"]["held_out_l1"]
    assert WL._seconds_to([(0.0, 0, 0.5), (1.0, 10, 0.3), (2.0, 20, 0.1)], 0.2) == 1.5
    assert WL._seconds_to([(0.0, 0, 0.5), (1.0, 10, 0.3)], 0.2) is None
