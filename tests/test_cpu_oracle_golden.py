"""The C oracle against golden vectors produced by the reference's own CUDA build
(tests/golden/make_ultragauss_golden.py run on a B200): bit-exact integer outputs,
images <= 1e-5 and gradients <= 1e-4 relative L2."""

from __future__ import annotations

import numpy as np
import pytest

from ug_helpers import golden_names, load_golden, rel_l2


@pytest.mark.parametrize("name", golden_names())
def test_oracle_matches_reference_golden(name):
    from oracle import ultragauss_oracle as O

    fx = load_golden(name)
    st = O.render(fx["means"], fx["precision_tril"], fx["opacities"], fx["intensities"], fx["pixels"], fx["geo"],
                  int(fx["H"]), int(fx["W"]), float(fx["chi2"]), float(fx["beta"]), bool(fx["sort_by_depth"]),
                  float(fx["bg_alpha"]), float(fx["bg_intensity"]))
    np.testing.assert_array_equal(st["touched"], fx["ref_touched"])
    vis = fx["ref_touched"] > 0
    np.testing.assert_array_equal(st["rects"][vis], fx["ref_rects"][vis])
    np.testing.assert_array_equal(st["keys"].astype(np.int64), fx["ref_keys"])
    np.testing.assert_array_equal(st["values"], fx["ref_values"])
    np.testing.assert_array_equal(st["range_start"], fx["ref_range_start"])
    np.testing.assert_array_equal(st["range_end"], fx["ref_range_end"])
    np.testing.assert_array_equal(st["counts"], fx["ref_counts"])
    np.testing.assert_array_equal(st["offsets"], fx["ref_offsets"])
    np.testing.assert_array_equal(st["indices"], fx["ref_indices"])
    for k in ("image", "alpha", "depth"):
        assert rel_l2(st[k], fx["ref_" + k]) <= 1e-5, k
    g = O.backward(st, fx["d_image"], fx["d_alpha"], fx["d_depth"])
    for k in ("d_means", "d_tril", "d_opacity", "d_intensity"):
        assert rel_l2(g[k], fx["ref_" + k]) <= 1e-4, k


def test_fp64_oracle_close_to_fp32():
    from oracle import ultragauss_oracle as O

    fx = load_golden("c1")
    args = (fx["means"], fx["precision_tril"], fx["opacities"], fx["intensities"], fx["pixels"], fx["geo"],
            int(fx["H"]), int(fx["W"]), float(fx["chi2"]), float(fx["beta"]), True, float(fx["bg_alpha"]), 0.0)
    a = O.render(*args)
    b = O.render(*args, precision="f64")
    assert rel_l2(a["image"], b["image"]) <= 1e-6
    ga = O.backward(a, fx["d_image"], fx["d_alpha"], fx["d_depth"])
    gb = O.backward(b, fx["d_image"], fx["d_alpha"], fx["d_depth"])
    for k in ga:
        assert rel_l2(ga[k], gb[k]) <= 1e-4, k
