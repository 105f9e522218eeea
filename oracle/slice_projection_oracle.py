"""TEST INFRASTRUCTURE ONLY: numpy restatement (float64) of the slice-adapted adapter's
projection of 3D Gaussians (baselines/slice_adapted_3dgs/render.py:66-98, 132-163) and of
its vector-Jacobian product written out by hand (the same chain rule the library's
us3d_sa_project_backward evaluates): view transform, camera covariance r^T R diag(s^2) R^T r,
slice sigma, cull, clamped 2x2 inverse, weights."""

from __future__ import annotations

import numpy as np


def _rot(qn):
    w, x, y, z = qn.T
    R = np.empty((qn.shape[0], 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z); R[:, 0, 1] = 2 * (x * y - z * w); R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w); R[:, 1, 1] = 1 - 2 * (x * x + z * z); R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w); R[:, 2, 1] = 2 * (y * z + x * w); R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def project(means, scales, quats, opac, colors, view, focal_depth, thickness, cull_std, thickness_scale, min_cov,
            normalize):
    m = np.asarray(means, np.float64)
    s = np.asarray(scales, np.float64)
    q = np.asarray(quats, np.float64)
    o = np.asarray(opac, np.float64).reshape(-1)
    V = np.asarray(view, np.float64)
    cam = m @ V[:3, :3] + V[3, :3]
    rel_z = cam[:, 2] - focal_depth
    qlen = np.linalg.norm(q, axis=1)
    qn = q / np.maximum(qlen, 1e-8)[:, None]
    R = _rot(qn)
    S = R @ (np.eye(3)[None] * (s * s)[:, None, :]) @ R.transpose(0, 2, 1)
    r = V[:3, :3]
    C = r.T[None] @ S @ r[None]
    c2 = C[:, :2, :2] + np.eye(2)[None] * min_cov
    var_raw = C[:, 2, 2]
    sigma = np.sqrt(np.maximum(var_raw, min_cov) + thickness ** 2)
    keep = np.abs(rel_z) <= cull_std * sigma * thickness_scale
    det_raw = c2[:, 0, 0] * c2[:, 1, 1] - c2[:, 0, 1] * c2[:, 1, 0]
    det = np.maximum(det_raw, min_cov)
    inv = np.stack([np.stack([c2[:, 1, 1] / det, -c2[:, 0, 1] / det], -1),
                    np.stack([-c2[:, 1, 0] / det, c2[:, 0, 0] / det], -1)], -2)
    u = rel_z / np.maximum(sigma, 1e-6)
    E = np.exp(-0.5 * u * u)
    w = o * E / (np.sqrt(det) if normalize else 1.0)
    st = dict(m=m, s=s, q=q, o=o, V=V, cam=cam, rel_z=rel_z, qlen=qlen, qn=qn, R=R, c2=c2, var_raw=var_raw,
              sigma=sigma, keep=keep, det_raw=det_raw, det=det, inv=inv, u=u, E=E, w=w, min_cov=min_cov,
              normalize=normalize)
    k = keep
    return dict(keep=keep, means2d=cam[k, :2], inv2d=inv[k], weights=w[k, None],
                colors=np.asarray(colors, np.float64)[k], state=st)


def project_backward(pr, d_means2d, d_inv2d, d_weights, d_colors, n_colors_rows):
    st = pr["state"]
    k = np.nonzero(st["keep"])[0]
    G = st["m"].shape[0]
    dm = np.zeros((G, 3)); ds = np.zeros((G, 3)); dq = np.zeros((G, 4)); dop = np.zeros(G)
    dc = np.zeros((n_colors_rows, 3))
    dc[k] = d_colors
    c2, det, det_raw = st["c2"][k], st["det"][k], st["det_raw"][k]
    sig, u, E, w, o = st["sigma"][k], st["u"][k], st["E"][k], st["w"][k], st["o"][k]
    szc = np.maximum(sig, 1e-6)
    dw = np.asarray(d_weights, np.float64).reshape(-1)
    nd = 1 / np.sqrt(det) if st["normalize"] else np.ones_like(det)
    dop[k] = dw * E * nd
    du = -dw * w * u
    drelz = du / szc
    dsig = np.where(sig >= 1e-6, -du * u / szc, 0.0)
    ddet = -0.5 * dw * w / det if st["normalize"] else np.zeros_like(det)
    di = np.asarray(d_inv2d, np.float64)
    ddet = ddet - (di[:, 0, 0] * c2[:, 1, 1] - di[:, 0, 1] * c2[:, 0, 1] - di[:, 1, 0] * c2[:, 1, 0]
                   + di[:, 1, 1] * c2[:, 0, 0]) / det ** 2
    dC = np.zeros((k.size, 3, 3))
    dC[:, 0, 0] = di[:, 1, 1] / det; dC[:, 1, 1] = di[:, 0, 0] / det
    dC[:, 0, 1] = -di[:, 0, 1] / det; dC[:, 1, 0] = -di[:, 1, 0] / det
    act = det_raw >= st["min_cov"]
    dC[:, 0, 0] += np.where(act, ddet * c2[:, 1, 1], 0); dC[:, 1, 1] += np.where(act, ddet * c2[:, 0, 0], 0)
    dC[:, 0, 1] -= np.where(act, ddet * c2[:, 1, 0], 0); dC[:, 1, 0] -= np.where(act, ddet * c2[:, 0, 1], 0)
    dC[:, 2, 2] = np.where(st["var_raw"][k] >= st["min_cov"], dsig * 0.5 / sig, 0)
    V = st["V"]
    dcam = np.concatenate([np.asarray(d_means2d, np.float64), drelz[:, None]], 1)
    dm[k] = dcam @ V[:3, :3].T
    r = V[:3, :3]
    dS = r[None] @ dC @ r.T[None]
    R = st["R"][k]
    s = st["s"][k]
    Dd = s * s
    dR = (dS + dS.transpose(0, 2, 1)) @ R * Dd[:, None, :]
    ds[k] = 2 * s * np.einsum("nik,nij,njk->nk", R, dS, R)
    qn = st["qn"][k]
    w_, x, y, z = qn.T
    gw = 2 * (-z * dR[:, 0, 1] + y * dR[:, 0, 2] + z * dR[:, 1, 0] - x * dR[:, 1, 2] - y * dR[:, 2, 0] + x * dR[:, 2, 1])
    gx = 2 * (y * dR[:, 0, 1] + z * dR[:, 0, 2] + y * dR[:, 1, 0] - 2 * x * dR[:, 1, 1] - w_ * dR[:, 1, 2]
              + z * dR[:, 2, 0] + w_ * dR[:, 2, 1] - 2 * x * dR[:, 2, 2])
    gy = 2 * (-2 * y * dR[:, 0, 0] + x * dR[:, 0, 1] + w_ * dR[:, 0, 2] + x * dR[:, 1, 0] + z * dR[:, 1, 2]
              - w_ * dR[:, 2, 0] + z * dR[:, 2, 1] - 2 * y * dR[:, 2, 2])
    gz = 2 * (-2 * z * dR[:, 0, 0] - w_ * dR[:, 0, 1] + x * dR[:, 0, 2] + w_ * dR[:, 1, 0] - 2 * z * dR[:, 1, 1]
              + y * dR[:, 1, 2] + x * dR[:, 2, 0] + y * dR[:, 2, 1])
    g = np.stack([gw, gx, gy, gz], 1)
    ql = st["qlen"][k]
    big = ql > 1e-8
    dot = (qn * g).sum(1, keepdims=True)
    dq[k] = np.where(big[:, None], (g - qn * dot) / np.where(big, ql, 1.0)[:, None], g * 1e8)
    return dict(d_means=dm, d_scales=ds, d_quats=dq, d_opacities=dop, d_colors=dc)
