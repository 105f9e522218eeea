"""TEST INFRASTRUCTURE ONLY: numpy/ctypes front end of the C oracle for UltraGauss.

``render`` runs the restated reference pipeline for one slice — mapper
(ops/ultragauss_renderer/src/mapper/wrapper_mapper.cu:35-206: project, scan, keys, stable
sort, ranges, per-pixel candidate CSR) and shader forward (src/shader/forward.cu:17-76);
``backward`` runs the adjoint (src/shader/backward.cu:17-131). ``precision`` selects the
fp32 restatement (reference arithmetic) or the fp64 oracle.

Parity of this restatement is pinned against outputs of the reference's own CUDA build
(oracle/_ref, run on a B200) stored as fixtures in tests/golden/.
"""

from __future__ import annotations

import ctypes
from ctypes import c_double, c_float, c_int, c_int32, c_int64, c_void_p
from pathlib import Path

import numpy as np

from . import build as _build

_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(str(_build.build()))
        for prec, real in (("f32", c_float), ("f64", c_double)):
            getattr(_lib, f"ugo_project_{prec}").argtypes = [c_int64, c_void_p, c_void_p, c_void_p, c_int, c_int, real,
                                                             real, c_void_p, c_void_p, c_void_p]
            getattr(_lib, f"ugo_keys_{prec}").argtypes = [c_int64, c_int, c_int, c_void_p, c_void_p, c_void_p,
                                                          c_void_p, c_void_p]
            getattr(_lib, f"ugo_pixel_candidates_{prec}").argtypes = [
                c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, real, real,
                c_void_p, c_void_p, c_void_p, c_void_p]
            getattr(_lib, f"ugo_forward_{prec}").argtypes = [
                c_int64, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                c_void_p, real, real, real, real, c_void_p, c_void_p, c_void_p]
            getattr(_lib, f"ugo_backward_{prec}").argtypes = [
                c_int64, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, real, real, real, real, c_void_p, c_void_p,
                c_void_p]
        _lib.ugo_sort_pairs.argtypes = [c_int64, c_int, c_void_p, c_void_p]
        _lib.ugo_tile_ranges.argtypes = [c_int64, c_void_p, c_int, c_void_p, c_void_p]
        _lib.ugo_set_threads.argtypes = [c_int]
        _lib.ugo_num_threads.restype = c_int
    return _lib


def set_threads(n: int) -> None:
    lib().ugo_set_threads(int(n))


def num_threads() -> int:
    return int(lib().ugo_num_threads())


def _p(a: np.ndarray):
    return a.ctypes.data_as(c_void_p)


def _arr(x, dtype):
    try:
        import torch

        if isinstance(x, torch.Tensor):
            x = x.detach().cpu().numpy()
    except ImportError:  # pragma: no cover
        pass
    return np.ascontiguousarray(np.asarray(x, dtype=dtype))


def geometry(origin, lat, ax, ele, lateral_spacing, axial_spacing, axial_near, col_offset, dtype=np.float32):
    return np.concatenate([_arr(origin, dtype).reshape(3), _arr(lat, dtype).reshape(3), _arr(ax, dtype).reshape(3),
                           _arr(ele, dtype).reshape(3),
                           np.array([lateral_spacing, axial_spacing, axial_near, col_offset], dtype=dtype)])


def render(means, tril, opac, inten, pixels, geo, H, W, chi2=7.815, beta=1e-4, sort_by_depth=True,
           bg_alpha=0.0, bg_intensity=0.0, precision="f32", want_indices=True, want_ambiguous=True):
    dt = np.float32 if precision == "f32" else np.float64
    L = lib()
    means = _arr(means, dt).reshape(-1, 3)
    tril = _arr(tril, dt).reshape(-1, 6)
    attr = np.stack([_arr(opac, dt).reshape(-1), _arr(inten, dt).reshape(-1)], axis=1).copy()
    pixels = _arr(pixels, dt).reshape(-1, 3)
    geo = _arr(geo, dt)
    G, P = means.shape[0], pixels.shape[0]
    tiles_x, tiles_y = (W + 15) // 16, (H + 15) // 16
    T = tiles_x * tiles_y
    touched = np.zeros(G, np.int32)
    rects = np.zeros((G, 4), np.int32)
    depths = np.zeros(G, dt)
    getattr(L, f"ugo_project_{precision}")(G, _p(means), _p(tril), _p(geo), H, W, chi2, beta, _p(touched),
                                            _p(rects), _p(depths))
    offsets = np.zeros(G + 1, np.int64)
    np.cumsum(touched, out=offsets[1:])
    n = int(offsets[-1])
    keys = np.zeros(n, np.uint64)
    vals = np.zeros(n, np.int32)
    getattr(L, f"ugo_keys_{precision}")(G, tiles_x, int(sort_by_depth), _p(rects), _p(depths), _p(offsets),
                                         _p(keys), _p(vals))
    unsorted_keys = keys.copy()
    L.ugo_sort_pairs(n, 0 if sort_by_depth else 32, _p(keys), _p(vals))
    rs = np.full(T, -1, np.int32)
    re = np.full(T, -1, np.int32)
    L.ugo_tile_ranges(n, _p(keys), T, _p(rs), _p(re))
    counts = np.zeros(P, np.int32)
    amb = np.zeros(P, np.int32)
    getattr(L, f"ugo_pixel_candidates_{precision}")(H, W, _p(pixels), _p(means), _p(tril), _p(vals), _p(rs), _p(re),
                                                     _p(geo), chi2, beta, _p(counts), None, None,
                                                     _p(amb) if want_ambiguous else None)
    poff = np.zeros(P + 1, np.int64)
    np.cumsum(counts, out=poff[1:])
    indices = np.zeros(int(poff[-1]), np.int32)
    getattr(L, f"ugo_pixel_candidates_{precision}")(H, W, _p(pixels), _p(means), _p(tril), _p(vals), _p(rs), _p(re),
                                                     _p(geo), chi2, beta, None, _p(poff), _p(indices), None)
    image = np.zeros(P, dt)
    alpha = np.zeros(P, dt)
    depth = np.zeros(P, dt)
    origin = geo[0:3].copy()
    ele = geo[9:12].copy()
    getattr(L, f"ugo_forward_{precision}")(P, G, _p(attr), _p(means), _p(tril), _p(pixels), _p(origin), _p(ele),
                                            _p(poff), _p(counts), _p(indices), bg_alpha, bg_intensity, chi2, beta,
                                            _p(image), _p(alpha), _p(depth))
    return {
        "touched": touched, "rects": rects, "depths": depths, "instance_offsets": offsets,
        "unsorted_keys": unsorted_keys, "keys": keys, "values": vals, "range_start": rs, "range_end": re,
        "counts": counts, "offsets": poff[:-1].astype(np.int32), "offsets64": poff, "indices": indices,
        "ambiguous": amb, "image": image, "alpha": alpha, "depth": depth,
        "_inputs": dict(means=means, tril=tril, attr=attr, pixels=pixels, geo=geo, chi2=chi2, beta=beta,
                        bg_alpha=bg_alpha, bg_intensity=bg_intensity, precision=precision),
    }


def backward(state, d_image, d_alpha, d_depth):
    inp = state["_inputs"]
    prec = inp["precision"]
    dt = np.float32 if prec == "f32" else np.float64
    L = lib()
    G = inp["means"].shape[0]
    P = inp["pixels"].shape[0]
    dI, dA, dD = (_arr(x, dt).reshape(-1) for x in (d_image, d_alpha, d_depth))
    dm = np.zeros((G, 4), dt)
    dtr = np.zeros((G, 6), dt)
    da = np.zeros((G, 2), dt)
    geo = inp["geo"]
    origin = geo[0:3].copy()
    ele = geo[9:12].copy()
    alpha = _arr(state["alpha"], dt)
    getattr(L, f"ugo_backward_{prec}")(P, G, _p(dI), _p(dA), _p(dD), _p(inp["attr"]), _p(inp["means"]),
                                        _p(inp["tril"]), _p(inp["pixels"]), _p(origin), _p(ele),
                                        _p(state["offsets64"]), _p(state["counts"]), _p(state["indices"]), _p(alpha),
                                        inp["bg_alpha"], inp["bg_intensity"], inp["chi2"], inp["beta"], _p(dm), _p(dtr),
                                        _p(da))
    return {"d_means": dm[:, :3].copy(), "d_tril": dtr, "d_opacity": da[:, 0].copy(), "d_intensity": da[:, 1].copy()}
