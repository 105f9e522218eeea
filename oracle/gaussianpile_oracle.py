"""TEST INFRASTRUCTURE ONLY: numpy/ctypes front end of the C oracle for GaussianPile
(restatement of ops/gaussianplie_renderer: core_tile.cu mapper, forward.cu tile additive
forward, us_focus.cu backward). Pinned against the reference's own CUDA build through the
fixtures in tests/golden/ (gaussianpile_*.npz)."""

from __future__ import annotations

from ctypes import c_double, c_float, c_int, c_int64, c_void_p

import numpy as np

from . import build as _build

_lib = None


def lib():
    global _lib
    if _lib is None:
        import ctypes

        _lib = ctypes.CDLL(str(_build.build()))
        for prec, real in (("f32", c_float), ("f64", c_double)):
            getattr(_lib, f"gpo_mapper_{prec}").argtypes = [c_int64] + [c_void_p] * 6 + [c_int, c_int, real, real, real,
                                                                                     c_int, real, c_void_p, c_void_p]
            getattr(_lib, f"gpo_tile_lists_{prec}").argtypes = [c_int64, c_void_p, c_int, c_int, c_void_p, c_void_p,
                                                                c_void_p]
            getattr(_lib, f"gpo_forward_{prec}").argtypes = [c_int64] + [c_void_p] * 8 + [c_int, c_int, c_int, real,
                                                                                       c_void_p, c_void_p, c_void_p,
                                                                                       c_void_p]
            getattr(_lib, f"gpo_backward_{prec}").argtypes = ([c_int64] + [c_void_p] * 8 + [c_int, c_int, c_int, real]
                                                              + [c_void_p] * 5 + [c_int] + [c_void_p] * 6)
    return _lib


def _a(x, dt):
    try:
        import torch

        if isinstance(x, torch.Tensor):
            x = x.detach().cpu().numpy()
    except ImportError:  # pragma: no cover
        pass
    return np.ascontiguousarray(np.asarray(x, dtype=dt))


def _p(a):
    return a.ctypes.data_as(c_void_p)


def render(means, scales, quats, opac, inten, pose, grid, params, H, W, lat_mm, ax_mm, near_mm, tile=16, k_sigma=3.0,
           precision="f32"):
    dt = np.float32 if precision == "f32" else np.float64
    L = lib()
    means, scales, quats = _a(means, dt).reshape(-1, 3), _a(scales, dt).reshape(-1, 3), _a(quats, dt).reshape(-1, 4)
    opac, inten = _a(opac, dt).reshape(-1), _a(inten, dt).reshape(-1)
    pose, grid, params = _a(pose, dt).reshape(16), _a(grid, dt).reshape(-1), _a(params, dt).reshape(-1)
    G = means.shape[0]
    tx, ty = (W + tile - 1) // tile, (H + tile - 1) // tile
    rects = np.zeros((G, 4), np.int32)
    touched = np.zeros(G, np.int32)
    getattr(L, f"gpo_mapper_{precision}")(G, _p(means), _p(scales), _p(quats), _p(pose), _p(grid), _p(params), H, W,
                                          lat_mm, ax_mm, near_mm, tile, k_sigma, _p(rects), _p(touched))
    n = int(touched.sum())
    rs = np.zeros(tx * ty, np.int32)
    re = np.zeros(tx * ty, np.int32)
    ids = np.zeros(max(n, 1), np.int32)
    getattr(L, f"gpo_tile_lists_{precision}")(G, _p(rects), tx, tx * ty, _p(rs), _p(re), _p(ids))
    image = np.zeros(H * W, dt)
    getattr(L, f"gpo_forward_{precision}")(G, _p(means), _p(scales), _p(quats), _p(opac), _p(inten), _p(pose), _p(grid),
                                           _p(params), H, W, tile, k_sigma, _p(rs), _p(re), _p(ids), _p(image))
    return {"rects": rects, "touched": touched, "sorted_ids": ids[:n], "range_start": rs, "range_end": re,
            "image": image.reshape(H, W),
            "_in": dict(means=means, scales=scales, quats=quats, opac=opac, inten=inten, pose=pose, grid=grid,
                        params=params, H=H, W=W, tile=tile, k_sigma=k_sigma, precision=precision, ids=ids)}


def backward(state, grad_image, pose_grad=False):
    i = state["_in"]
    dt = np.float32 if i["precision"] == "f32" else np.float64
    G = i["means"].shape[0]
    gi = _a(grad_image, dt).reshape(-1)
    out = dict(d_means=np.zeros((G, 3), dt), d_scales=np.zeros((G, 3), dt), d_quats=np.zeros((G, 4), dt),
               d_opacity=np.zeros(G, dt), d_intensity=np.zeros(G, dt), d_pose=np.zeros(16, dt))
    getattr(lib(), f"gpo_backward_{i['precision']}")(
        G, _p(i["means"]), _p(i["scales"]), _p(i["quats"]), _p(i["opac"]), _p(i["inten"]), _p(i["pose"]),
        _p(i["grid"]), _p(i["params"]), i["H"], i["W"], i["tile"], i["k_sigma"], _p(state["rects"]),
        _p(state["range_start"]), _p(state["range_end"]), _p(i["ids"]), _p(gi), int(pose_grad), _p(out["d_means"]),
        _p(out["d_scales"]), _p(out["d_quats"]), _p(out["d_opacity"]), _p(out["d_intensity"]), _p(out["d_pose"]))
    out["d_pose"] = out["d_pose"].reshape(4, 4)
    return out
