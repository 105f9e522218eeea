"""TEST INFRASTRUCTURE ONLY: numpy/ctypes front end of the slice-adapted 3DGS C oracle
(restatement of ops/slice_adapted_3dgs_renderer/src/render.cu's bounded splat)."""

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
            getattr(_lib, f"sao_bin_{prec}").argtypes = [c_int64, c_int, c_int, real, real, c_void_p, c_void_p, real,
                                                         c_void_p, c_void_p, c_void_p, c_void_p, c_int64]
            getattr(_lib, f"sao_bin_{prec}").restype = c_int64
            getattr(_lib, f"sao_forward_{prec}").argtypes = [c_int, c_int, real, real] + [c_void_p] * 4 + [real] + [
                c_void_p] * 5
            getattr(_lib, f"sao_backward_{prec}").argtypes = [c_int64, c_int, c_int, real, real] + [c_void_p] * 4 + [
                real] + [c_void_p] * 9
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


def render(H, W, hw, hh, means2d, inv2d, weights, colors, radius_sigma=3.0, precision="f32"):
    dt = np.float32 if precision == "f32" else np.float64
    L = lib()
    m, iv = _a(means2d, dt).reshape(-1, 2), _a(inv2d, dt).reshape(-1, 4)
    w, c = _a(weights, dt).reshape(-1), _a(colors, dt).reshape(-1, 3)
    N = m.shape[0]
    T = ((W + 15) // 16) * ((H + 15) // 16)
    bbox = np.zeros((N, 4), np.int32)
    rs = np.zeros(T, np.int32)
    re = np.zeros(T, np.int32)
    total = getattr(L, f"sao_bin_{precision}")(N, H, W, hw, hh, _p(m), _p(iv), radius_sigma, _p(bbox), _p(rs), _p(re),
                                                None, 0)
    ids = np.zeros(max(total, 1), np.int32)
    getattr(L, f"sao_bin_{precision}")(N, H, W, hw, hh, _p(m), _p(iv), radius_sigma, _p(bbox), _p(rs), _p(re), _p(ids),
                                       total)
    image = np.zeros((H * W, 3), dt)
    alpha = np.zeros(H * W, dt)
    getattr(L, f"sao_forward_{precision}")(H, W, hw, hh, _p(m), _p(iv), _p(w), _p(c), radius_sigma, _p(rs), _p(re),
                                           _p(ids), _p(image), _p(alpha))
    return {"sorted_ids": ids[:total], "range_start": rs, "range_end": re, "image": image, "alpha": alpha[:, None],
            "_in": (H, W, hw, hh, m, iv, w, c, radius_sigma, precision, ids)}


def backward(state, grad_image, grad_alpha):
    H, W, hw, hh, m, iv, w, c, rs_, prec, ids = state["_in"]
    dt = np.float32 if prec == "f32" else np.float64
    N = m.shape[0]
    gi, ga = _a(grad_image, dt).reshape(-1, 3), _a(grad_alpha, dt).reshape(-1)
    dm, di, dw, dc = np.zeros((N, 2), dt), np.zeros((N, 2, 2), dt), np.zeros((N, 1), dt), np.zeros((N, 3), dt)
    getattr(lib(), f"sao_backward_{prec}")(N, H, W, hw, hh, _p(m), _p(iv), _p(w), _p(c), rs_, _p(state["range_start"]),
                                           _p(state["range_end"]), _p(ids), _p(gi), _p(ga), _p(dm), _p(di), _p(dw),
                                           _p(dc))
    return {"d_means": dm, "d_inv": di, "d_weights": dw, "d_colors": dc}
