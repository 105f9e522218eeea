"""The GaussianPile C oracle against golden vectors from the reference's own CUDA build."""

from __future__ import annotations

import numpy as np
import pytest

from gp_helpers import gp_golden_names, load_gp
from ug_helpers import rel_l2


@pytest.mark.parametrize("name", gp_golden_names())
def test_gaussianpile_oracle_matches_reference_golden(name):
    from oracle import gaussianpile_oracle as GO

    fx = load_gp(name)
    m = fx["meta"].tolist()
    st = GO.render(fx["means"], fx["scales"], fx["quats"], fx["opacities"], fx["intensities"], fx["pose"], fx["grid"],
                   fx["params"], int(fx["H"]), int(fx["W"]), m[2], m[3], m[4], int(m[5]), m[8])
    vis = fx["ref_rects"][:, 0] < fx["ref_rects"][:, 2]
    np.testing.assert_array_equal(st["rects"][vis], fx["ref_rects"][vis])
    np.testing.assert_array_equal(st["sorted_ids"], fx["ref_sorted_ids"])
    np.testing.assert_array_equal(st["range_start"], fx["ref_range_start"])
    np.testing.assert_array_equal(st["range_end"], fx["ref_range_end"])
    assert rel_l2(st["image"], fx["ref_image"]) <= 1e-5
    g = GO.backward(st, fx["grad_image"], pose_grad=bool(fx["pose_grad"]))
    for k in ("d_means", "d_opacity", "d_intensity"):
        assert rel_l2(g[k], fx["ref_" + k]) <= 1e-4, (k, rel_l2(g[k], fx["ref_" + k]))
    for k in ("d_scales", "d_quats"):  # fp32 finite differences of the adjoint (see the GPU tests)
        assert rel_l2(g[k], fx["ref_" + k]) <= 5e-3, (k, rel_l2(g[k], fx["ref_" + k]))
    if int(fx["pose_grad"]):
        assert rel_l2(g["d_pose"], fx["ref_d_pose"]) <= 2e-3
