"""TEST INFRASTRUCTURE ONLY: numpy/ctypes front end of the UltraGray C oracle
(restatement of ops/ultragray_renderer's mapper and shader)."""

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
            f = getattr(_lib, f"ugro_map_{prec}")
            f.argtypes = [c_int64, c_int] + [c_void_p] * 6 + [real] * 5 + [c_void_p] * 4 + [c_int64]
            f.restype = c_int64
            f = getattr(_lib, f"ugro_forward_{prec}")
            f.argtypes = [c_int, c_int] + [c_void_p] * 14 + [real, real, c_int, real, c_void_p, c_void_p]
            f.restype = None
            f = getattr(_lib, f"ugro_backward_{prec}")
            f.argtypes = [c_int64, c_int, c_int] + [c_void_p] * 14 + [real, real, c_int, real] + [c_void_p] * 7
            f.restype = None
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


def render(scene: dict, precision: str = "f32") -> dict:
    """scene keys: means (G,3), scales (G,3), quats (G,4), attenuations (G), sh (G,4),
    pixels (W,H,3), ray_o (W,3), ray_d (W,3), origin, lat, ele, ax (3), pert (W), and the
    floats width_mm, near_mm, col_off, elev_cut, k_sigma, wr, local (bool), maxwin."""
    dt = np.float32 if precision == "f32" else np.float64
    L = lib()
    a = {k: _a(scene[k], dt) for k in ("means", "scales", "quats", "attenuations", "sh", "pixels", "ray_o", "ray_d",
                                        "origin", "lat", "ele", "ax", "pert")}
    G = a["means"].shape[0]
    W, H = a["pixels"].shape[0], a["pixels"].shape[1]
    counts = np.zeros(W, np.int32)
    offsets = np.zeros(W, np.int32)
    mp = getattr(L, f"ugro_map_{precision}")
    args = (G, W, _p(a["means"]), _p(a["scales"]), _p(a["origin"]), _p(a["lat"]), _p(a["ele"]), _p(a["ax"]),
            scene["width_mm"], scene["near_mm"], scene["col_off"], scene["elev_cut"], scene["k_sigma"])
    total = mp(*args, _p(counts), _p(offsets), None, None, 0)
    idx = np.zeros(max(total, 1), np.int32)
    depths = np.zeros(max(total, 1), dt)
    mp(*args, _p(counts), _p(offsets), _p(idx), _p(depths), total)
    image = np.zeros((H, W), dt)
    state = np.zeros((W, H, 4), dt)
    getattr(L, f"ugro_forward_{precision}")(
        W, H, _p(counts), _p(offsets), _p(idx), _p(depths), _p(a["means"]), _p(a["scales"]), _p(a["quats"]),
        _p(a["attenuations"]), _p(a["sh"]), _p(a["pixels"]), _p(a["ray_o"]), _p(a["ray_d"]), _p(a["ele"]),
        _p(a["pert"]), scene["k_sigma"], scene["wr"], 1 if scene.get("local", False) else 0,
        scene.get("maxwin", 17.0), _p(image), _p(state))
    return dict(a=a, dt=dt, precision=precision, G=G, W=W, H=H, counts=counts, offsets=offsets,
                indices=idx[:total], depths=depths[:total], total=int(total), image=image, state=state,
                scene=scene, _idx=idx, _depths=depths)


def backward(st: dict, grad_image) -> dict:
    L = lib()
    a, dt, G = st["a"], st["dt"], st["G"]
    sc = st["scene"]
    gi = _a(grad_image, dt).reshape(st["H"], st["W"])
    dm = np.zeros((G, 3), dt)
    ds = np.zeros((G, 3), dt)
    dq = np.zeros((G, 4), dt)
    da = np.zeros(G, dt)
    dsh = np.zeros((G, 4), dt)
    getattr(L, f"ugro_backward_{st['precision']}")(
        G, st["W"], st["H"], _p(st["counts"]), _p(st["offsets"]), _p(st["_idx"]), _p(st["_depths"]), _p(a["means"]),
        _p(a["scales"]), _p(a["quats"]), _p(a["attenuations"]), _p(a["sh"]), _p(a["pixels"]), _p(a["ray_o"]),
        _p(a["ray_d"]), _p(a["ele"]), _p(a["pert"]), sc["k_sigma"], sc["wr"], 1 if sc.get("local", False) else 0,
        sc.get("maxwin", 17.0), _p(st["state"]), _p(gi), _p(dm), _p(ds), _p(dq), _p(da), _p(dsh))
    return dict(d_means=dm, d_scales=ds, d_quats=dq, d_attens=da, d_sh=dsh)
