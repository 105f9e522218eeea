"""Seeded synthetic scenes and probe sweeps (the real ultrasound datasets are not available
offline; these stand in with the distributions the workloads are specified by).

Headline scene: G anisotropic Gaussians in a 64 mm cube, means uniform, per-axis
log-scales N(log 1.0 mm, 0.3), uniformly random unit quaternions, intensity U(0,1),
opacity sigmoid(N(0,1)). Frames: planar B-mode slices from a linear sweep (probe moved
along the elevational axis, tilt N(0, 2 deg) about the lateral axis). All draws come from
one ``torch.Generator`` in a fixed order.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List

import torch


@dataclass
class GaussianScene:
    means: torch.Tensor  # (G,3)
    scales: torch.Tensor  # (G,3)
    quats: torch.Tensor  # (G,4) wxyz, unit
    opacities: torch.Tensor  # (G,)
    intensities: torch.Tensor  # (G,)
    precision_tril: torch.Tensor  # (G,6) raw factor, l11,l12,l13,l22,l23,l33

    def to(self, device) -> "GaussianScene":
        return GaussianScene(*(getattr(self, f).to(device) for f in
                               ("means", "scales", "quats", "opacities", "intensities", "precision_tril")))


@dataclass
class Slice:
    height: int
    width: int
    lateral_spacing: float
    axial_spacing: float
    axial_near: float
    lateral_col_offset: float
    origin: torch.Tensor
    axis_lat: torch.Tensor
    axis_ax: torch.Tensor
    axis_ele: torch.Tensor
    pixels: torch.Tensor  # (H*W, 3) world positions of pixel centres

    def to(self, device) -> "Slice":
        return Slice(self.height, self.width, self.lateral_spacing, self.axial_spacing, self.axial_near,
                     self.lateral_col_offset, *(getattr(self, f).to(device) for f in
                                                ("origin", "axis_lat", "axis_ax", "axis_ele", "pixels")))


def quat_to_rot(q: torch.Tensor) -> torch.Tensor:
    """Rotation matrices of unit (w,x,y,z) quaternions."""
    w, x, y, z = q.unbind(-1)
    return torch.stack(
        [
            1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
            2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
            2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y),
        ],
        dim=-1,
    ).reshape(*q.shape[:-1], 3, 3)


def precision_tril_from_scales_quats(scales: torch.Tensor, quats: torch.Tensor, beta: float = 1e-4) -> torch.Tensor:
    """Raw lower-Cholesky factor of Lambda = R diag(1/s^2) R^T with diagonal raw^2 + beta
    (the parameterisation UltraGauss learns); computed in float64 with elementwise operations
    only, written out for 3x3 matrices: batched BLAS / LAPACK kernels may round differently
    from run to run (buffer alignment, threads), which would make the scenes, and results that
    sit on a threshold, differ between processes."""
    s = scales.double().clamp_min(beta)
    R = quat_to_rot(quats.double())
    inv = 1.0 / (s * s)

    def lam(i, j):  # Lambda_ij = sum_k R_ik R_jk / s_k^2
        return (R[:, i, 0] * R[:, j, 0] * inv[:, 0] + R[:, i, 1] * R[:, j, 1] * inv[:, 1]
                + R[:, i, 2] * R[:, j, 2] * inv[:, 2])

    a00, a10, a20, a11, a21, a22 = lam(0, 0), lam(1, 0), lam(2, 0), lam(1, 1), lam(2, 1), lam(2, 2)
    l00 = a00.sqrt()
    l10 = a10 / l00
    l20 = a20 / l00
    l11 = (a11 - l10 * l10).sqrt()
    l21 = (a21 - l20 * l10) / l11
    l22 = (a22 - l20 * l20 - l21 * l21).sqrt()

    def raw(d):
        return (d - beta).clamp_min(1e-8).sqrt()

    return torch.stack([raw(l00), l10, l20, raw(l11), l21, raw(l22)], dim=1).float()


def make_scene(n: int, seed: int = 0, cube_mm: float = 64.0, log_scale_mean: float = 0.0,
               log_scale_std: float = 0.3, opacity_mu: float = 0.0, opacity_std: float = 1.0,
               beta: float = 1e-4) -> GaussianScene:
    # The transcendental functions and the quaternion norm run in float64 on elementwise
    # operations and are rounded to float32 once: CPU kernels evaluate exp / sigmoid / norms with
    # vector and scalar code paths whose last bits differ, and which elements take which path can
    # change from process to process.
    g = torch.Generator().manual_seed(seed)
    means = torch.rand((n, 3), generator=g) * cube_mm
    scales64 = torch.exp(log_scale_mean + log_scale_std * torch.randn((n, 3), generator=g).double())
    q = torch.randn((n, 4), generator=g).double()
    q = q / (q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1] + q[:, 2] * q[:, 2] + q[:, 3] * q[:, 3]).sqrt().clamp_min(1e-12)[:, None]
    intensities = torch.rand((n,), generator=g)
    opacities = torch.sigmoid(opacity_mu + opacity_std * torch.randn((n,), generator=g).double()).float()
    tril = precision_tril_from_scales_quats(scales64, q, beta)
    return GaussianScene(means, scales64.float(), q.float(), opacities, intensities, tril)


def slice_pixels(origin, lat, ax, H, W, lateral_spacing, axial_spacing, axial_near, col_offset) -> torch.Tensor:
    """Pixel-centre world positions, row-major (row = axial), as the reference pipeline
    builds them (pipeline_god_file.py:299-306)."""
    u = torch.arange(W, dtype=torch.float32)
    v = torch.arange(H, dtype=torch.float32)
    lateral_mm = (u - col_offset) * lateral_spacing
    axial_mm = axial_near + v * axial_spacing
    yy, xx = torch.meshgrid(axial_mm, lateral_mm, indexing="ij")
    pix = origin.view(1, 1, 3) + xx[..., None] * lat.view(1, 1, 3) + yy[..., None] * ax.view(1, 1, 3)
    return pix.reshape(-1, 3).contiguous()


def _rot_about(axis: torch.Tensor, angle: float) -> torch.Tensor:
    axis = axis / axis.norm()
    x, y, z = axis.tolist()
    c, s = math.cos(angle), math.sin(angle)
    C = 1 - c
    return torch.tensor([[c + x * x * C, x * y * C - z * s, x * z * C + y * s],
                         [y * x * C + z * s, c + y * y * C, y * z * C - x * s],
                         [z * x * C - y * s, z * y * C + x * s, c + z * z * C]], dtype=torch.float32)


def linear_sweep(n_frames: int, H: int, W: int, spacing_mm: float, seed: int = 0, cube_mm: float = 64.0,
                 step_mm: float = 2.0, tilt_deg: float = 2.0) -> List[Slice]:
    """Probe translated ``step_mm`` per frame along elevation through the cube centre,
    each frame tilted about its lateral axis by N(0, tilt_deg)."""
    g = torch.Generator().manual_seed(seed + 1_000_003)
    tilts = torch.randn((n_frames,), generator=g) * math.radians(tilt_deg)
    out = []
    col_off = (W - 1) * 0.5
    depth_mm = H * spacing_mm
    for f in range(n_frames):
        z = cube_mm * 0.5 + (f - (n_frames - 1) * 0.5) * step_mm
        lat0 = torch.tensor([1.0, 0.0, 0.0])
        ax0 = torch.tensor([0.0, 1.0, 0.0])
        ele0 = torch.tensor([0.0, 0.0, 1.0])
        R = _rot_about(lat0, float(tilts[f]))
        ax = R @ ax0
        ele = R @ ele0
        centre = torch.tensor([cube_mm * 0.5, cube_mm * 0.5, z])
        origin = centre - ax * (depth_mm * 0.5)
        pix = slice_pixels(origin, lat0, ax, H, W, spacing_mm, spacing_mm, 0.0, col_off)
        out.append(Slice(H, W, spacing_mm, spacing_mm, 0.0, col_off, origin, lat0.clone(), ax, ele, pix))
    return out


def _unit_quaternions(n: int, g: torch.Generator) -> torch.Tensor:
    q = torch.randn((n, 4), generator=g).double()
    return q / (q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1] + q[:, 2] * q[:, 2] + q[:, 3] * q[:, 3]).sqrt().clamp_min(1e-12)[:, None]


def make_clustered_scene(n: int, seed: int = 0, extent_mm=(100.0, 60.0, 80.0), n_clusters: int = 20,
                         background: float = 0.1, log_scale_mean: float = math.log(0.8), log_scale_std: float = 0.4,
                         opacity_mu: float = -1.0, opacity_std: float = 1.0, semi_axes_mm=(3.0, 12.0),
                         beta: float = 1e-4) -> GaussianScene:
    """Tissue-like scene: ``n`` Gaussians in a box of ``extent_mm``, a mixture of
    ``n_clusters`` ellipsoidal clusters plus a fraction ``background`` drawn uniformly in the
    box. Cluster c has a centre uniform in the inner 80 % of the box, semi-axes U(semi_axes_mm)
    and a random orientation; its members are uniform inside the ellipsoid (clamped to the
    box). Per Gaussian: log-scales N(log_scale_mean, log_scale_std), random unit quaternions,
    intensity U(0,1), opacity sigmoid(N(opacity_mu, opacity_std)).

    Draw order from one generator: cluster centres, semi-axes, orientations; the cluster of
    every clustered Gaussian; its direction and radius in the unit ball; the background means;
    then scales, quaternions, intensities and opacities as in make_scene."""
    g = torch.Generator().manual_seed(seed)
    ext = torch.tensor(extent_mm, dtype=torch.float64)
    n_bg = int(round(background * n))
    n_cl = n - n_bg
    centres = (0.1 + 0.8 * torch.rand((n_clusters, 3), generator=g).double()) * ext
    lo, hi = semi_axes_mm
    semi = lo + (hi - lo) * torch.rand((n_clusters, 3), generator=g).double()
    rot = quat_to_rot(_unit_quaternions(n_clusters, g))
    which = torch.randint(0, n_clusters, (n_cl,), generator=g)
    d = torch.randn((n_cl, 3), generator=g).double()
    d = d / (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2]).sqrt().clamp_min(1e-12)[:, None]
    r = torch.rand((n_cl,), generator=g).double().pow(1.0 / 3.0)
    local = d * r[:, None] * semi[which]
    Rw = rot[which]  # elementwise products: no batched BLAS, whose rounding can vary between processes
    pts = centres[which] + torch.stack([Rw[:, i, 0] * local[:, 0] + Rw[:, i, 1] * local[:, 1]
                                        + Rw[:, i, 2] * local[:, 2] for i in range(3)], dim=1)
    pts = torch.minimum(torch.maximum(pts, torch.zeros(3, dtype=torch.float64)), ext)
    bg = torch.rand((n_bg, 3), generator=g).double() * ext
    means = torch.cat([pts, bg]).float().contiguous()
    scales64 = torch.exp(log_scale_mean + log_scale_std * torch.randn((n, 3), generator=g).double())
    q = _unit_quaternions(n, g)
    intensities = torch.rand((n,), generator=g)
    opacities = torch.sigmoid(opacity_mu + opacity_std * torch.randn((n,), generator=g).double()).float()
    tril = precision_tril_from_scales_quats(scales64, q, beta)
    return GaussianScene(means, scales64.float(), q.float(), opacities, intensities, tril)


def _axis_angle(axis: torch.Tensor, angle: float) -> torch.Tensor:
    """Rotation matrix (float64) about a unit axis (Rodrigues)."""
    x, y, z = (float(v) for v in axis)
    K = torch.tensor([[0.0, -z, y], [z, 0.0, -x], [-y, x, 0.0]], dtype=torch.float64)
    return torch.eye(3, dtype=torch.float64) + math.sin(angle) * K + (1.0 - math.cos(angle)) * (K @ K)


def random_walk_sweep(n_frames: int, H: int, W: int, spacing_mm: float, seed: int = 0,
                      extent_mm=(100.0, 60.0, 80.0), step_mm: float = 1.5, step_deg: float = 1.0) -> List[Slice]:
    """Freehand-like sweep: the probe pose is a cumulative random walk, each frame moved by
    ``step_mm`` along a random direction and turned by ``step_deg`` about a random axis
    (both uniform on the sphere) from the previous one. The first frame stands in the middle
    of the box: lateral axis x, axial axis y (depth from the box's top face), elevation z,
    the image centred laterally and its top row ``(extent_y - H * spacing) / 2`` below the
    top face. Pixel centres as slice_pixels (column offset (W - 1) / 2)."""
    g = torch.Generator().manual_seed(seed + 2_000_003)
    ext = torch.tensor(extent_mm, dtype=torch.float64)
    R = torch.eye(3, dtype=torch.float64)  # columns: lateral, axial, elevational axes
    depth = H * spacing_mm
    origin = torch.tensor([ext[0] * 0.5, max(0.0, (float(ext[1]) - depth) * 0.5), ext[2] * 0.5], dtype=torch.float64)
    col_off = (W - 1) * 0.5
    out = []
    for f in range(n_frames):
        if f > 0:
            t = torch.randn((3,), generator=g).double()
            a = torch.randn((3,), generator=g).double()
            origin = origin + step_mm * t / t.norm().clamp_min(1e-12)
            R = _axis_angle(a / a.norm().clamp_min(1e-12), math.radians(step_deg)) @ R
        lat, ax, ele = (R[:, i].float().contiguous() for i in range(3))
        o = origin.float()
        pix = slice_pixels(o, lat, ax, H, W, spacing_mm, spacing_mm, 0.0, col_off)
        out.append(Slice(H, W, spacing_mm, spacing_mm, 0.0, col_off, o, lat, ax, ele, pix))
    return out


# Attenuation of the B-mode workload: 0.5 dB/cm/MHz at 5 MHz, two-way (echo path), i.e.
# 0.5 dB per mm of depth.
BMODE_DB_PER_MM = 2.0 * 0.5 * 5.0 / 10.0


def bmode_attenuation_logit(n_gauss: int, volume_mm3: float, sigma_mm: float = 1.0, window_mm: float = 2.0,
                            db_per_mm: float = BMODE_DB_PER_MM) -> float:
    """Attenuation logit tau_raw of the ray-integral renderer that makes a scene of n_gauss
    Gaussians in volume_mm3 attenuate like tissue of db_per_mm.

    The renderer multiplies, for every Gaussian a ray has passed, T = tau + (1 - tau) e^-psi,
    tau = sigmoid(tau_raw), psi the integral of the Gaussian's profile along the ray over its
    quadrature window. A ray meets on average rho * 2 pi sigma^2 Gaussians of scale sigma per
    mm of depth (rho = n_gauss / volume_mm3), so each stands for delta = 1 / (rho 2 pi sigma^2)
    mm of tissue and should transmit T* = 10^(-db_per_mm delta / 20) on a central crossing,
    where psi0 = sqrt(2 pi) sigma erf(window / (sigma sqrt 2)). Solving for tau gives the
    logit. It only sets inputs; the renderer's arithmetic is the reference's."""
    rho = n_gauss / volume_mm3
    delta = 1.0 / (rho * 2.0 * math.pi * sigma_mm * sigma_mm)
    t_star = 10.0 ** (-db_per_mm * delta / 20.0)
    psi0 = math.sqrt(2.0 * math.pi) * sigma_mm * math.erf(window_mm / (sigma_mm * math.sqrt(2.0)))
    e0 = math.exp(-psi0)
    tau = (t_star - e0) / (1.0 - e0)
    return math.log(tau / (1.0 - tau))


@dataclass
class BModeScene:
    means: torch.Tensor        # (G,3)
    scales: torch.Tensor       # (G,3)
    quats: torch.Tensor        # (G,4) wxyz, unit
    attenuations: torch.Tensor  # (G,) logits
    sh: torch.Tensor           # (G,4) degree-1 echo coefficients (reflectivity c0, c1..c3)

    def to(self, device) -> "BModeScene":
        return BModeScene(*(getattr(self, f).to(device) for f in ("means", "scales", "quats", "attenuations", "sh")))


def make_bmode_scene(n: int, seed: int = 0, aperture_mm: float = 40.0, depth_mm: float = 60.0,
                     sweep_mm: float = 64.0, log_scale_mean: float = 0.0, log_scale_std: float = 0.3,
                     strong_fraction: float = 0.05, window_mm: float = 2.0) -> BModeScene:
    """Scene of the ray-integral B-mode workload: n Gaussians uniform in a box of
    aperture_mm (lateral, x) x depth_mm (axial, y) x sweep_mm (elevation, z); per-axis
    log-scales N(log_scale_mean, log_scale_std) (1 mm median), random unit quaternions;
    reflectivity c0 ~ U(0, 1) with a fraction strong_fraction of strong reflectors U(5, 10),
    c1..c3 = 0; attenuation logits from bmode_attenuation_logit (0.5 dB/cm/MHz at 5 MHz).
    Draw order: means, log-scales, quaternions, reflectivity, strong-reflector choice and value."""
    g = torch.Generator().manual_seed(seed)
    ext = torch.tensor([aperture_mm, depth_mm, sweep_mm])
    means = torch.rand((n, 3), generator=g) * ext
    scales64 = torch.exp(log_scale_mean + log_scale_std * torch.randn((n, 3), generator=g).double())
    q = _unit_quaternions(n, g)
    refl = torch.rand((n,), generator=g)
    strong = torch.rand((n,), generator=g) < strong_fraction
    strong_val = 5.0 + 5.0 * torch.rand((n,), generator=g)
    refl = torch.where(strong, strong_val, refl)
    sh = torch.zeros((n, 4))
    sh[:, 0] = refl
    logit = bmode_attenuation_logit(n, float(ext.prod()), sigma_mm=math.exp(log_scale_mean), window_mm=window_mm)
    att = torch.full((n,), logit, dtype=torch.float32)
    return BModeScene(means.contiguous(), scales64.float(), q.float(), att, sh)


@dataclass
class ScanlineFrame:
    """One B-mode frame of a linear array: W scanlines of H samples."""
    origin: torch.Tensor      # (3,) probe origin (centre of the array face)
    axis_lat: torch.Tensor
    axis_ax: torch.Tensor
    axis_ele: torch.Tensor
    width_mm: float           # aperture
    depth_mm: float
    ray_origins: torch.Tensor  # (W,3)
    ray_dirs: torch.Tensor     # (W,3)
    pixels: torch.Tensor       # (W,H,3) sample positions, ray-major
    col_offset: float


def bmode_sweep(n_frames: int, W: int = 512, H: int = 1024, aperture_mm: float = 40.0, depth_mm: float = 60.0,
                sweep_mm: float = 64.0) -> List[ScanlineFrame]:
    """Linear array translated along the elevational axis through the box of make_bmode_scene
    (frames evenly spaced over sweep_mm): lateral axis x, axial axis y (depth), elevation z;
    scanline x at lateral offset (x - (W-1)/2) * aperture / W from the array centre, samples
    at depths (y + 0.5) * depth / H."""
    out = []
    lat = torch.tensor([1.0, 0.0, 0.0])
    ax = torch.tensor([0.0, 1.0, 0.0])
    ele = torch.tensor([0.0, 0.0, 1.0])
    col_off = (W - 1) * 0.5
    spacing = aperture_mm / W
    xs = (torch.arange(W, dtype=torch.float64) - col_off) * spacing
    zs = (torch.arange(H, dtype=torch.float64) + 0.5) * (depth_mm / H)
    for f in range(n_frames):
        z = (f + 0.5) * sweep_mm / n_frames
        o = torch.tensor([aperture_mm * 0.5, 0.0, z], dtype=torch.float64)
        ro = o[None, :] + xs[:, None] * lat.double()[None, :]
        pix = ro[:, None, :] + zs[None, :, None] * ax.double()[None, None, :]
        out.append(ScanlineFrame(o.float(), lat.clone(), ax.clone(), ele.clone(), aperture_mm, depth_mm,
                                 ro.float().contiguous(), ax.repeat(W, 1).contiguous(), pix.float().contiguous(),
                                 col_off))
    return out
