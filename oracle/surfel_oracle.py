"""TEST INFRASTRUCTURE ONLY: numpy/ctypes front end of the UltraGS-baseline surfel C oracle
(restatement of ops/ultrags_baseline_renderer/cuda_rasterizer)."""

from __future__ import annotations

import ctypes
from ctypes import c_double, c_float, c_int, c_int64, c_void_p

import numpy as np

from . import build as _build

_lib = None
_structs = {}


def _struct(real):
    if real not in _structs:
        class GsIn(ctypes.Structure):
            _fields_ = [("P", c_int), ("D", c_int), ("M", c_int), ("W", c_int), ("H", c_int), ("scale_modifier", real),
                        ("means", c_void_p), ("shs", c_void_p), ("colors", c_void_p), ("opac", c_void_p),
                        ("scales", c_void_p), ("rots", c_void_p), ("transmat", c_void_p), ("view", c_void_p),
                        ("proj", c_void_p), ("campos", c_void_p), ("bg", c_void_p)]
        _structs[real] = GsIn
    return _structs[real]


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(str(_build.build()))
        for prec, real in (("f32", c_float), ("f64", c_double)):
            S = ctypes.POINTER(_struct(real))
            f = getattr(_lib, f"gso_bin_{prec}")
            f.argtypes = [S, c_void_p, c_void_p, c_void_p, c_int64, c_void_p]
            f.restype = c_int64
            f = getattr(_lib, f"gso_forward_{prec}")
            f.argtypes = [S] + [c_void_p] * 7
            f.restype = None
            f = getattr(_lib, f"gso_backward_{prec}")
            f.argtypes = [S] + [c_void_p] * 8 + [c_float, c_float] + [c_void_p] * 8
            f.restype = None
    return _lib


def _a(x, dt):
    return np.ascontiguousarray(np.asarray(x, dtype=dt))


def _p(a):
    return None if a is None or a.size == 0 else a.ctypes.data_as(c_void_p)


def render(scene: dict, precision: str = "f32") -> dict:
    """scene: the dict of tests/gs_helpers.make_scene (empty arrays for absent inputs)."""
    dt = np.float32 if precision == "f32" else np.float64
    real = c_float if precision == "f32" else c_double
    L = lib()
    keep = {k: _a(scene[k], dt) for k in ("means", "shs", "colors", "opacities", "scales", "quats", "transmat",
                                          "viewmatrix", "projmatrix", "campos", "bg")}
    P = keep["means"].shape[0]
    precomp = keep["transmat"].size > 0
    M = keep["shs"].shape[1] if keep["shs"].size else 0
    W, H = int(scene["W"]), int(scene["H"])
    s = _struct(real)(P, int(scene["sh_degree"]), M, W, H, float(scene["scale_modifier"]), _p(keep["means"]),
                      _p(keep["shs"]), _p(keep["colors"]), _p(keep["opacities"]),
                      None if precomp else _p(keep["scales"]), None if precomp else _p(keep["quats"]),
                      _p(keep["transmat"]), _p(keep["viewmatrix"]), _p(keep["projmatrix"]), _p(keep["campos"]),
                      _p(keep["bg"]))
    T = ((W + 15) // 16) * ((H + 15) // 16)
    radii = np.zeros(P, np.int32)
    recs = np.zeros((max(P, 1), 20), dt)
    ranges = np.zeros((T, 2), np.int32)
    sb = ctypes.byref(s)
    fb = getattr(L, f"gso_bin_{precision}")
    total = fb(sb, _p(radii), recs.ctypes.data_as(c_void_p), None, 0, None)
    pl = np.zeros(max(total, 1), np.int32)
    fb(sb, _p(radii), recs.ctypes.data_as(c_void_p), pl.ctypes.data_as(c_void_p), total,
       ranges.ctypes.data_as(c_void_p))
    color = np.zeros((3, H, W), dt)
    others = np.zeros((7, H, W), dt)
    accum = np.zeros((3, H, W), dt)
    nc = np.zeros((2, H, W), np.uint32)
    getattr(L, f"gso_forward_{precision}")(sb, recs.ctypes.data_as(c_void_p), pl.ctypes.data_as(c_void_p),
                                           ranges.ctypes.data_as(c_void_p), color.ctypes.data_as(c_void_p),
                                           others.ctypes.data_as(c_void_p), accum.ctypes.data_as(c_void_p),
                                           nc.ctypes.data_as(c_void_p))
    return dict(struct=s, keep=keep, dt=dt, precision=precision, P=P, M=M, W=W, H=H, num=int(total), radii=radii,
                recs=recs, point_list=pl[:total], ranges=ranges, color=color, others=others, accum=accum,
                n_contrib=nc, _pl=pl, scene=scene, precomp=precomp)


def backward(st: dict, grad_color, grad_others) -> dict:
    L = lib()
    dt, P, M = st["dt"], st["P"], st["M"]
    gc = _a(grad_color, dt)
    go = _a(grad_others, dt)
    out = dict(d_means2D=np.zeros((P, 3), dt), d_colors=np.zeros((P, 3), dt), d_opacity=np.zeros((P, 1), dt),
               d_means3D=np.zeros((P, 3), dt), d_transmat=np.zeros((P, 9), dt), d_sh=np.zeros((P, M, 3), dt),
               d_scales=np.zeros((P, 2), dt), d_rot=np.zeros((P, 4), dt))
    sc = st["scene"]
    v = lambda k: out[k].ctypes.data_as(c_void_p)  # noqa: E731
    getattr(L, f"gso_backward_{st['precision']}")(
        ctypes.byref(st["struct"]), st["recs"].ctypes.data_as(c_void_p), st["radii"].ctypes.data_as(c_void_p),
        st["_pl"].ctypes.data_as(c_void_p), st["ranges"].ctypes.data_as(c_void_p), st["accum"].ctypes.data_as(c_void_p),
        st["n_contrib"].ctypes.data_as(c_void_p), gc.ctypes.data_as(c_void_p), go.ctypes.data_as(c_void_p),
        float(sc["tanfovx"]), float(sc["tanfovy"]), v("d_means2D"), v("d_colors"), v("d_opacity"), v("d_means3D"),
        v("d_transmat"), v("d_sh") if M else None, None if st["precomp"] else v("d_scales"),
        None if st["precomp"] else v("d_rot"))
    return out
