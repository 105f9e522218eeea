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

    out = WL.run_training(n_init=20_000, n_gt=40_000, n_frames=48, size=128, spacing_mm=0.5, batch=8, steps=60,
                          refine_every=20, plain_frames=64, max_gaussians=40_000, device=cuda_device)
    b = out["batched"]
    assert b["frames"] == 480 and b["frames_per_s"] > 0
    assert len(b["refinements"]) == 3
    assert b["held_out_l1"] < out["held_out_l1_at_start"], out
    assert 0.0 < out["plain"]["held_out_l1"] < 1.0
