"""The slice-adapted projection restatement and its hand-written VJP against golden vectors
made by the reference adapter's own PyTorch code (autograd for the gradients)."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from ug_helpers import rel_l2

GOLDEN = Path(__file__).resolve().parent / "golden"
NAMES = sorted(p.stem.split("_", 2)[2] for p in GOLDEN.glob("slice_projection_*.npz"))


def load(name):
    return dict(np.load(GOLDEN / f"slice_projection_{name}.npz"))


def args(d):
    return (d["means"], d["scales"], d["quats"], d["opacities"], d["colors"], d["view"], float(d["focal_depth"]),
            float(d["set_slice_thickness_mm"]), float(d["set_cull_std"]), float(d["set_thickness_scale"]),
            float(d["set_min_covariance"]), bool(d["set_normalize_by_footprint"]))


@pytest.mark.parametrize("name", NAMES)
def test_projection_oracle_matches_reference_golden(name):
    from oracle import slice_projection_oracle as PO

    d = load(name)
    pr = PO.project(*args(d))
    np.testing.assert_array_equal(pr["keep"], d["ref_keep"])
    for k in ("means2d", "inv2d", "weights", "colors"):
        assert rel_l2(pr[k], d["ref_" + k]) <= 1e-5, (k, rel_l2(pr[k], d["ref_" + k]))
    g = PO.project_backward(pr, d["up_means2d"], d["up_inv2d"], d["up_weights"], d["up_colors"], d["colors"].shape[0])
    for k in ("means", "scales", "quats", "opacities", "colors"):
        r = d["ref_d_" + k]
        assert rel_l2(g["d_" + k].reshape(r.shape), r) <= 1e-4, (k, rel_l2(g["d_" + k].reshape(r.shape), r))
