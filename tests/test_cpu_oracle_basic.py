"""Self-checks of the C oracle's building blocks against independent numpy / pure-Python
statements of the same rules (small sizes)."""

from __future__ import annotations

import numpy as np


def test_stable_radix_sort_matches_numpy_stable():
    from oracle import ultragauss_oracle as O

    rng = np.random.default_rng(0)
    n = 5000
    tiles = rng.integers(0, 40, n).astype(np.uint64)
    depth = rng.integers(0, 50, n).astype(np.uint64)  # many ties
    keys = (tiles << np.uint64(32)) | depth
    vals = np.arange(n, dtype=np.int32)
    for begin in (0, 32):
        k = keys.copy()
        v = vals.copy()
        O.lib().ugo_sort_pairs(n, begin, O._p(k), O._p(v))
        order = np.argsort(keys >> np.uint64(begin), kind="stable")
        np.testing.assert_array_equal(v, vals[order])
        np.testing.assert_array_equal(k, keys[order])


def test_tile_ranges_rule():
    from oracle import ultragauss_oracle as O

    keys = (np.array([0, 0, 2, 2, 2, 5], dtype=np.uint64) << np.uint64(32))
    rs = np.zeros(7, np.int32)
    re = np.zeros(7, np.int32)
    O.lib().ugo_tile_ranges(len(keys), O._p(keys), 7, O._p(rs), O._p(re))
    np.testing.assert_array_equal(rs, [0, -1, 2, -1, -1, 5, -1])
    np.testing.assert_array_equal(re, [2, -1, 5, -1, -1, 6, -1])


def _py_radii(t, chi2, beta, axis):
    l11, l12, l13, l22, l23, l33 = t[0] ** 2 + beta, t[1], t[2], t[3] ** 2 + beta, t[4], t[5] ** 2 + beta
    y0 = axis[0] / max(l11, 1e-10)
    y1 = (axis[1] - l12 * y0) / max(l22, 1e-10)
    y2 = (axis[2] - l13 * y0 - l23 * y1) / max(l33, 1e-10)
    return max(1e-3, np.sqrt(chi2) * np.sqrt(max(y0 * y0 + y1 * y1 + y2 * y2, 1e-12)))


def test_window_radius_is_chi2_extent():
    """r = sqrt(chi2 * a^T Sigma a) with Sigma = (L L^T)^-1 (the ellipsoid's extent on a)."""
    rng = np.random.default_rng(1)
    for _ in range(20):
        t = rng.normal(0, 1, 6) + np.array([1.2, 0, 0, 1.1, 0, 0.9])
        L = np.array([[t[0] ** 2 + 1e-4, 0, 0], [t[1], t[3] ** 2 + 1e-4, 0], [t[2], t[4], t[5] ** 2 + 1e-4]])
        sigma = np.linalg.inv(L @ L.T)
        a = rng.normal(size=3)
        a /= np.linalg.norm(a)
        r = _py_radii(t, 7.815, 1e-4, a)
        assert abs(r - np.sqrt(7.815 * a @ sigma @ a)) <= 1e-9 * max(r, 1)


def test_oracle_forward_matches_python_loop():
    """Tiny scene: the oracle's per-pixel forward equals a direct double-precision loop over
    the reference's candidate rule (tile list + window test, chi2 cut, 1e-8 skip)."""
    import torch

    from oracle import ultragauss_oracle as O
    from us3d_b200 import scenes

    sc = scenes.make_scene(40, seed=3, cube_mm=12.0, log_scale_mean=0.4)
    fr = scenes.linear_sweep(3, 20, 24, 0.5, seed=3, cube_mm=12.0)[1]
    geo = O.geometry(fr.origin, fr.axis_lat, fr.axis_ax, fr.axis_ele, 0.5, 0.5, 0.0, fr.lateral_col_offset,
                     dtype=np.float64)
    st = O.render(sc.means, sc.precision_tril, sc.opacities, sc.intensities, fr.pixels, geo, 20, 24, 7.815, 1e-4,
                  True, 0.01, 0.2, precision="f64")
    m = sc.means.double().numpy()
    t = sc.precision_tril.double().numpy()
    o = sc.opacities.double().numpy()
    c = sc.intensities.double().numpy()
    pix = fr.pixels.double().numpy()
    lat, ax, ele = geo[3:6], geo[6:9], geo[9:12]
    for p in range(0, 480, 7):
        tile = (p // 24 // 16) * 2 + (p % 24) // 16
        s, e = st["range_start"][tile], st["range_end"][tile]
        sa = sc_ = 0.0
        if s >= 0:
            for g in st["values"][s:e]:
                d = pix[p] - m[g]
                if not (abs(d @ lat) <= _py_radii(t[g], 7.815, 1e-4, lat) and abs(d @ ax) <= _py_radii(t[g], 7.815, 1e-4, ax)):
                    continue
                L = np.array([[t[g][0] ** 2 + 1e-4, 0, 0], [t[g][1], t[g][3] ** 2 + 1e-4, 0],
                              [t[g][2], t[g][4], t[g][5] ** 2 + 1e-4]])
                q = d @ (L @ L.T) @ d
                if q > 7.815:
                    continue
                ah = o[g] * np.exp(-0.5 * q)
                if ah <= 1e-8:
                    continue
                sa += ah
                sc_ += ah * c[g]
        img = min(1.0, max(0.0, (sc_ + 0.01 * 0.2) / max(sa + 0.01, 1e-8)))
        assert abs(img - st["image"][p]) <= 1e-12, p
        assert abs(sa + 0.01 - st["alpha"][p]) <= 1e-12, p
