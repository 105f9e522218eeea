"""Slice grid pack: 16 floats describing a linear probe's pixel grid on the device.

The reference imports ``build_slice_grid_pack`` and ``shader_weight_mode_id`` from a package
(``ours_renderer.grid_geometry``) that is not part of its tree; this module provides them
with the layout its kernels read (ops/gaussianplie_renderer/include/shader/
slice_grid_geometry.cuh:4-24): [0] probe type (0 = linear), [1] H, [2] W, [3] lateral
spacing (mm/px), [4] axial spacing (mm/px), [5] near (mm), [6] lateral column offset,
[7] centre-lateral flag, [8] radius (mm, convex), [9] field of view (deg, convex),
[10..15] unused.
"""

from __future__ import annotations

import torch

SLICE_GRID_PACK_LEN = 16
_SHADER_WEIGHT_MODES = {"probe3d": 0, "plane_cond2d": 1, "us_focus": 2}


def shader_weight_mode_id(name) -> int:
    """Numeric id of a shader weight mode name ("probe3d", "plane_cond2d", "us_focus")."""
    if isinstance(name, int):
        return int(name)
    key = str(name).strip().lower()
    if key not in _SHADER_WEIGHT_MODES:
        raise ValueError(f"unknown shader weight mode {name!r}; expected one of {sorted(_SHADER_WEIGHT_MODES)}")
    return _SHADER_WEIGHT_MODES[key]


def build_slice_grid_pack(meta, device=None) -> torch.Tensor:
    """Pack for a linear probe from an object with H, W, delta_lateral_mm, delta_axial_mm,
    near_mm and center_lateral (the lateral column offset is (W-1)/2 when centred, else 0)."""
    H = int(getattr(meta, "H"))
    W = int(getattr(meta, "W"))
    centre = bool(getattr(meta, "center_lateral", True))
    pack = torch.zeros(SLICE_GRID_PACK_LEN, dtype=torch.float32)
    pack[0] = 0.0
    pack[1] = float(H)
    pack[2] = float(W)
    pack[3] = float(getattr(meta, "delta_lateral_mm"))
    pack[4] = float(getattr(meta, "delta_axial_mm"))
    pack[5] = float(getattr(meta, "near_mm", 0.0))
    pack[6] = float(W - 1) * 0.5 if centre else 0.0
    pack[7] = 1.0 if centre else 0.0
    return pack.to(device) if device is not None else pack


__all__ = ["build_slice_grid_pack", "shader_weight_mode_id", "SLICE_GRID_PACK_LEN"]
