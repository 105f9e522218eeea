"""Helpers for the UltraGS-baseline surfel rasteriser tests: seeded camera scenes, the
reference's own build run on them (with its geometry / binning / image byte buffers decoded),
and one B200 render + backward through the library."""

from __future__ import annotations

import math
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"

SCENE_ARRAYS = ("means", "scales", "quats", "opacities", "shs", "colors", "transmat", "viewmatrix", "projmatrix",
                "campos", "bg", "grad_color", "grad_others")
SCENE_SCALARS = ("W", "H", "tanfovx", "tanfovy", "scale_modifier", "sh_degree")


def _proj(znear, zfar, tanfovx, tanfovy):
    top, right = tanfovy * znear, tanfovx * znear
    P = np.zeros((4, 4))
    P[0, 0] = 2.0 * znear / (2 * right)
    P[1, 1] = 2.0 * znear / (2 * top)
    P[3, 2] = 1.0
    P[2, 2] = zfar / (zfar - znear)
    P[2, 3] = -(zfar * znear) / (zfar - znear)
    return P


def make_scene(P, W, H, seed, sh_degree=0, mode="sh", fovx_deg=55.0, yaw=0.2, scale_range=(0.02, 0.25),
               scale_modifier=1.0):
    """mode: 'sh' (SH colours of the given degree), 'colors' (precomputed colours),
    'transmat' (precomputed homographies are filled in by the caller from a first run)."""
    rng = np.random.default_rng(seed)
    tanfovx = math.tan(math.radians(fovx_deg) / 2)
    tanfovy = tanfovx * H / W
    # camera at c, rotated by yaw about y, looking along its +z
    c = np.array([0.3, -0.2, -1.0])
    cy, sy = math.cos(yaw), math.sin(yaw)
    Rcw = np.array([[cy, 0, -sy], [0, 1, 0], [sy, 0, cy]])  # world -> camera rotation
    V = np.eye(4)
    V[:3, :3] = Rcw
    V[:3, 3] = -Rcw @ c
    full = _proj(0.01, 100.0, tanfovx, tanfovy) @ V
    z = rng.uniform(1.5, 9.0, P)
    x = rng.uniform(-1.15, 1.15, P) * z * tanfovx
    y = rng.uniform(-1.15, 1.15, P) * z * tanfovy
    pc = np.stack([x, y, z], 1)
    pc[: max(1, P // 50), 2] = rng.uniform(-1.0, 0.15, max(1, P // 50))  # some behind the near plane
    means = (Rcw.T @ pc.T).T + c
    scales = np.exp(rng.uniform(np.log(scale_range[0]), np.log(scale_range[1]), (P, 2)))
    quats = rng.normal(size=(P, 4))
    opac = 1 / (1 + np.exp(-rng.normal(0.5, 1.2, (P, 1))))
    M = {0: 1, 1: 4, 2: 9, 3: 16}[sh_degree]
    shs = rng.normal(0.2, 0.6, (P, M, 3))
    colors = rng.uniform(0, 1, (P, 3))
    f = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
    return dict(means=f(means), scales=f(scales), quats=f(quats), opacities=f(opac),
                shs=f(shs) if mode == "sh" else f(np.zeros((0,))),
                colors=f(colors) if mode == "colors" else f(np.zeros((0,))),
                transmat=f(np.zeros((0,))), viewmatrix=f(V.T), projmatrix=f(full.T), campos=f(c),
                bg=f(rng.uniform(0, 1, 3)), grad_color=f(rng.normal(size=(3, H, W))),
                grad_others=f(rng.normal(size=(7, H, W))), W=int(W), H=int(H), tanfovx=float(tanfovx),
                tanfovy=float(tanfovy), scale_modifier=float(scale_modifier), sh_degree=int(sh_degree), mode=mode)


def _t(scene, k, dev):
    import torch

    return torch.as_tensor(scene[k]).to(dev).contiguous()


def decode_reference_buffers(geom, binning, img, P, R, W, H):
    """The reference's byte buffers laid out by GeometryState / BinningState / ImageState
    (cuda_rasterizer/rasterizer_impl.cu:142-183; 128-byte aligned chunks)."""
    g, b, im = geom.cpu().numpy(), binning.cpu().numpy(), img.cpu().numpy()

    def take(buf, off, dtype, count):
        off = (off + 127) // 128 * 128
        n = np.dtype(dtype).itemsize * count
        return np.frombuffer(buf[off:off + n].tobytes(), dtype=dtype).copy(), off + n

    o = 0
    depths, o = take(g, o, np.float32, P)
    clamped, o = take(g, o, np.bool_, 3 * P)
    radii, o = take(g, o, np.int32, P)
    means2d, o = take(g, o, np.float32, 2 * P)
    transmat, o = take(g, o, np.float32, 9 * P)
    normal_opacity, o = take(g, o, np.float32, 4 * P)
    rgb, o = take(g, o, np.float32, 3 * P)
    N = W * H
    o = 0
    accum, o = take(im, o, np.float32, 3 * N)
    n_contrib, o = take(im, o, np.uint32, 2 * N)
    ranges, o = take(im, o, np.uint32, 2 * N)
    o = 0
    point_list, o = take(b, o, np.uint32, R)
    _, o = take(b, o, np.uint32, R)
    keys, o = take(b, o, np.uint64, R)
    T = ((W + 15) // 16) * ((H + 15) // 16)
    return dict(depths=depths, clamped=clamped.reshape(P, 3), radii_internal=radii, means2d=means2d.reshape(P, 2),
                transmat=transmat.reshape(P, 9), normal_opacity=normal_opacity.reshape(P, 4), rgb=rgb.reshape(P, 3),
                accum=accum.reshape(3, H, W), n_contrib=n_contrib.reshape(2, H, W),
                ranges=ranges.reshape(N, 2)[:T], point_list=point_list, keys=keys)


def _args(scene, dev):
    import torch

    t = {}
    for k in SCENE_ARRAYS:
        t[k] = torch.empty(0, device=dev) if scene[k].size == 0 else _t(scene, k, dev)
    return t


def run_reference_gs(ref, scene, dev):
    """RasterizeGaussiansCUDA + RasterizeGaussiansBackwardCUDA of the reference build."""
    import torch

    t = _args(scene, dev)
    W, H = scene["W"], scene["H"]
    op = t["opacities"]
    # absent inputs are fresh empty tensors (NULL data pointers), as the reference's Python
    # front end passes them; prefiltered stays False (the reference traps the GPU otherwise)
    precomp = scene["transmat"].size > 0
    sc = torch.empty(0, device=dev) if precomp else t["scales"]
    rot = torch.empty(0, device=dev) if precomp else t["quats"]
    num, color, others, radii, gb, bb, ib = ref.rasterize_gaussians(
        t["bg"], t["means"], t["colors"], op, sc, rot, scene["scale_modifier"], t["transmat"], t["viewmatrix"],
        t["projmatrix"], scene["tanfovx"], scene["tanfovy"], H, W, t["shs"], scene["sh_degree"], t["campos"], False,
        False)
    grads = ref.rasterize_gaussians_backward(
        t["bg"], t["means"], radii, t["colors"], sc, rot, scene["scale_modifier"], t["transmat"], t["viewmatrix"],
        t["projmatrix"], scene["tanfovx"], scene["tanfovy"], t["grad_color"], t["grad_others"], t["shs"],
        scene["sh_degree"], t["campos"], gb, num, bb, ib, False)
    torch.cuda.synchronize()
    c = lambda x: x.detach().cpu().numpy()  # noqa: E731
    P = scene["means"].shape[0]
    out = dict(ref_num=np.int64(num), ref_color=c(color), ref_others=c(others), ref_radii=c(radii))
    names = ("d_means2D", "d_colors", "d_opacity", "d_means3D", "d_transmat", "d_sh", "d_scales", "d_rot")
    for k, v in zip(names, grads):
        out["ref_" + k] = c(v)
    st = decode_reference_buffers(gb, bb, ib, P, int(num), W, H)
    for k, v in st.items():
        out["ref_state_" + k] = v
    return out


def run_b200_gs(scene, dev, capacity=None, backward=True):
    import torch

    from us3d_b200 import surfel as S

    t = _args(scene, dev)
    precomp = scene["transmat"].size > 0
    sc = None if precomp else t["scales"]
    rot = None if precomp else t["quats"]
    num, color, others, radii, state = S.forward(t["bg"], t["means"], t["colors"], t["opacities"].reshape(-1), sc,
                                                  rot, scene["scale_modifier"], t["transmat"], t["viewmatrix"],
                                                  t["projmatrix"], scene["H"], scene["W"], t["shs"],
                                                  scene["sh_degree"], t["campos"], False, capacity=capacity)
    out = dict(num=num, color=color, others=others, radii=radii)
    if state is not None:
        pl, keys, ranges, nc, acc, rec = S.export(state)
        out.update(point_list=pl, keys=keys, ranges=ranges, n_contrib=nc, accum=acc, records=rec)
    if backward:
        g = S.backward(state, t["bg"], t["means"], radii, t["colors"], sc, rot, scene["scale_modifier"], t["transmat"],
                       t["viewmatrix"], t["projmatrix"], scene["tanfovx"], scene["tanfovy"], t["grad_color"],
                       t["grad_others"], t["shs"], scene["sh_degree"], t["campos"])
        for k, v in zip(("d_means2D", "d_colors", "d_opacity", "d_means3D", "d_transmat", "d_sh", "d_scales", "d_rot"),
                        g):
            out[k] = v
    torch.cuda.synchronize()
    return {k: (v.detach().cpu().numpy() if hasattr(v, "detach") else v) for k, v in out.items()}


def gs_golden_names():
    return sorted(p.stem.split("_", 1)[1] for p in GOLDEN.glob("ultrags_*.npz"))


def load_gs(name):
    p = GOLDEN / f"ultrags_{name}.npz"
    if not p.exists():
        import pytest

        pytest.skip(f"golden fixture {p.name} not generated")
    d = dict(np.load(p))
    scene = {k: d[k] for k in SCENE_ARRAYS}
    for k in SCENE_SCALARS:
        scene[k] = d[k].item()
    scene["mode"] = str(d["mode"])
    return scene, {k: v for k, v in d.items() if k.startswith("ref_")}


GS_GRADS = ("d_means2D", "d_colors", "d_opacity", "d_means3D", "d_transmat", "d_sh", "d_scales", "d_rot")

# name: (P, W, H, seed, make_scene arguments); 'transmat' cases reuse the homographies the
# reference computed for the same scene as precomputed inputs
CASES = {
    "deg0": (3000, 96, 80, 0, dict(sh_degree=0)),
    "deg2": (2000, 70, 50, 1, dict(sh_degree=2, scale_modifier=1.3)),
    "colors": (2500, 64, 64, 2, dict(mode="colors")),
    "transmat": (1500, 80, 48, 3, dict(sh_degree=1, mode="transmat")),
}


def build_case(ref, name, dev, P=None, W=None, H=None, seed=None, **kw):
    """The scene of a named case (or of explicit sizes) plus the reference's results."""
    if name in CASES:
        P, W, H, seed, kw = CASES[name]
    mode = kw.get("mode", "sh")
    scene = make_scene(P, W, H, seed, **{**kw, "mode": "sh" if mode == "transmat" else mode})
    if mode == "transmat":
        first = run_reference_gs(ref, scene, dev)
        scene["transmat"] = np.ascontiguousarray(first["ref_state_transmat"], dtype=np.float32)
        scene["mode"] = "transmat"
    return scene, run_reference_gs(ref, scene, dev)
