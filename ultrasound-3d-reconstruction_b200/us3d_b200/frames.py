"""Frame batches built on the device from a dataset held in device memory.

The reference's loader (``NpzUltrasoundDataset``, pipeline_god_file.py:172-336) reads one frame
per training step on the host: it scales 8-bit images to [0, 1], normalises the probe axes,
generates (or reads) the pixel centre positions, the scanlines (ray origins and directions) and
the world-to-probe pose, and copies everything to the GPU. Here the dataset is moved to the
device once (images kept in their stored 8-bit or float form, axes normalised with the
reference's ``_normalize``), and a batch of frames is assembled by one launch
(``us3d_frames_gather``) from a device tensor of dataset indices: frame records, pixel positions
(gathered, or generated bit-identically to the reference's grid) and targets;
``us3d_frames_geometry`` adds the scanlines and poses of the same indices.
"""

from __future__ import annotations

from typing import Optional

import numpy as np
import torch

from . import _lib
from . import ultragauss as UG
from .ultragauss import _ptr, _stream


def _normalize(x: torch.Tensor) -> torch.Tensor:
    """The reference's axis normalisation (pipeline_god_file.py:336-337), per frame."""
    return x / torch.clamp(torch.linalg.norm(x, dim=-1, keepdim=True), min=1.0e-8)


class DeviceFrameSource:
    """A dataset of N equally sized frames on the device, batched by ``fill``/``batch``.

    images: (N,H,W) or (N,1,H,W), uint8 or float (scaled by 1/255 when the maximum exceeds 1.5,
    as the reference does); origin, axis_lat, axis_ax, axis_ele: (N,3) or (3,) (axes are
    normalised per frame); pixel_positions: optional (N,H*W,3) or (N,H,W,3) mm, otherwise
    generated from the geometry with ``delta_lateral_mm``, ``delta_axial_mm``, ``near_mm`` and
    the lateral centring of the reference's config; ray_origins / ray_dirs: optional (N,W,3) and
    poses_world_to_probe optional (N,4,4), otherwise generated as the reference does. The UltraGS
    camera fields (pipeline_god_file.py:236-241): viewmatrix / projmatrix optional (N,4,4) or one
    (4,4) for all frames (identity when absent), camera_center optional (N,3) or (3,) (the frame's
    probe origin when absent), tanfovx / tanfovy optional (N,) or scalars (``default_tanfov``,
    the reference config's 0.5, when absent)."""

    def __init__(self, images, origin, axis_lat, axis_ax, axis_ele, delta_lateral_mm: float,
                 delta_axial_mm: float, near_mm: float = 0.0, center_lateral: bool = True,
                 pixel_positions=None, device: Optional[torch.device] = None, ray_origins=None, ray_dirs=None,
                 poses_world_to_probe=None, viewmatrix=None, projmatrix=None, camera_center=None, tanfovx=None,
                 tanfovy=None, default_tanfov=(0.5, 0.5)):
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        img = torch.as_tensor(np.asarray(images) if not torch.is_tensor(images) else images)
        if img.ndim == 4:
            img = img[:, 0]
        if img.ndim != 3:
            raise ValueError("images must be (N,H,W) or (N,1,H,W)")
        self.n, self.height, self.width = (int(x) for x in img.shape)
        if self.n == 0:
            raise ValueError("the dataset has no frames")
        self.images = (img if img.dtype == torch.uint8 else img.float()).contiguous().to(dev)
        scale = float(self.images.max()) > 1.5
        if img.dtype == torch.uint8:
            self.image_format = _lib.IMAGES_U8_DIV255 if scale else _lib.IMAGES_U8
        else:
            self.image_format = _lib.IMAGES_F32_DIV255 if scale else _lib.IMAGES_F32

        def per_frame(a, default):
            t = torch.as_tensor(np.asarray(a, dtype=np.float32) if a is not None else np.asarray(default, np.float32))
            t = t.reshape(-1, 3) if t.ndim >= 2 and t.shape[0] == self.n else t.reshape(1, 3).expand(self.n, 3)
            return t.to(dev, torch.float32).contiguous()

        o = per_frame(origin, [0.0, 0.0, 0.0])
        lat = _normalize(per_frame(axis_lat, [1.0, 0.0, 0.0]))
        ax = _normalize(per_frame(axis_ax, [0.0, 1.0, 0.0]))
        ele = _normalize(per_frame(axis_ele, [0.0, 0.0, 1.0]))
        col_off = (self.width - 1) * 0.5 if center_lateral else 0.0
        scal = torch.tensor([delta_lateral_mm, delta_axial_mm, near_mm, col_off], dtype=torch.float32)
        ints = torch.zeros(8, dtype=torch.int32)
        ints[:2] = torch.tensor([self.height, self.width], dtype=torch.int32)
        tail = torch.cat([scal, ints.view(torch.float32)]).to(dev).expand(self.n, 12)
        self.records = torch.cat([o, lat, ax, ele, tail], dim=1).contiguous()  # (N, 24) us3d_slice_frame
        self.pixel_positions = None
        if pixel_positions is not None:
            pp = torch.as_tensor(np.asarray(pixel_positions, dtype=np.float32))
            self.pixel_positions = pp.reshape(self.n, self.height * self.width, 3).to(dev).contiguous()
        def stored(a, shape):
            if a is None:
                return None
            return torch.as_tensor(np.asarray(a, dtype=np.float32)).reshape(self.n, *shape).to(dev).contiguous()

        self.ray_origins = stored(ray_origins, (self.width, 3))
        self.ray_dirs = stored(ray_dirs, (self.width, 3))
        self.poses = stored(poses_world_to_probe, (16,))

        def matrices(a):
            if a is None:
                return torch.eye(4, dtype=torch.float32).expand(self.n, 4, 4).to(dev).contiguous()
            m = torch.as_tensor(np.asarray(a, dtype=np.float32))
            m = m if (m.ndim == 3 and m.shape[0] == self.n) else m.reshape(1, 4, 4).expand(self.n, 4, 4)
            return m.to(dev).contiguous()

        def scalars(a, default):
            v = torch.as_tensor(np.asarray(a if a is not None else default, dtype=np.float32))
            v = v.reshape(-1) if (v.ndim >= 1 and v.shape[0] == self.n) else v.reshape(1).expand(self.n)
            return v.to(dev).contiguous()

        self.viewmatrix = matrices(viewmatrix)
        self.projmatrix = matrices(projmatrix)
        # camera centre: stored values, else the probe origin as stored (not normalised)
        self.camera_center = per_frame(camera_center, [0.0, 0.0, 0.0]) if camera_center is not None else o
        self.tanfovx = scalars(tanfovx, default_tanfov[0])
        self.tanfovy = scalars(tanfovy, default_tanfov[1])
        self.device = dev
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)

    @classmethod
    def from_npz(cls, path, delta_lateral_mm: float, delta_axial_mm: float, near_mm: float = 0.0,
                 center_lateral: bool = True, device: Optional[torch.device] = None) -> "DeviceFrameSource":
        """Loads the reference's NPZ layout (DATA_FORMAT.md of the reference: ``images`` and the
        optional per-frame geometry and pixel positions)."""
        raw = np.load(path, allow_pickle=False)
        get = (lambda k: raw[k] if k in raw else None)
        n = raw["images"].shape[0]
        pose = get("pose_world_to_probe")
        if pose is not None and not (pose.ndim == 3 and pose.shape[0] == n):
            pose = np.tile(np.asarray(pose, np.float32).reshape(1, 4, 4), (n, 1, 1))  # one pose for all
        return cls(raw["images"], get("probe_origin_world"), get("axis_lateral_world"), get("axis_axial_world"),
                   get("axis_elevational_world"), delta_lateral_mm, delta_axial_mm, near_mm, center_lateral,
                   get("pixel_positions_world"), device, get("ray_origins"), get("ray_dirs"), pose,
                   get("viewmatrix"), get("projmatrix"), get("camera_center"), get("tanfovx"), get("tanfovy"))

    def frame_table(self, batch_size: int) -> UG.FrameTable:
        """An (unfilled) frame table for batches of ``batch_size`` frames."""
        tx, ty = (self.width + 15) // 16, (self.height + 15) // 16
        hw = self.height * self.width
        return UG.FrameTable(torch.zeros((batch_size, 24), dtype=torch.float32, device=self.device), batch_size,
                             batch_size * tx * ty, batch_size * hw, [k * tx * ty for k in range(batch_size)],
                             [tx * ty] * batch_size, [k * hw for k in range(batch_size)],
                             [(self.height, self.width)] * batch_size)

    def fill(self, indices: torch.Tensor, table: UG.FrameTable, pixels: torch.Tensor, targets: torch.Tensor) -> None:
        """Writes the batch of dataset ``indices`` (device int64) into ``table``, ``pixels``
        (F*H*W, 3) and ``targets`` (F*H*W,) in place (one launch, no synchronisation)."""
        F = int(indices.numel())
        if table.n_frames != F or pixels.shape != (F * self.height * self.width, 3) or \
                targets.shape != (F * self.height * self.width,):
            raise ValueError("batch buffers do not match the number of indices")
        if indices.dtype != torch.int64 or indices.device != self.device:
            raise ValueError("indices must be an int64 tensor on the dataset's device")
        _lib.check(_lib.call("us3d_frames_gather", _ptr(self.records), self.n, _ptr(indices.contiguous()), F,
                             self.height, self.width, _ptr(self.pixel_positions), _ptr(self.images),
                             self.image_format, _ptr(table.table), _ptr(pixels), _ptr(targets), _ptr(self.status),
                             _stream()), "us3d_frames_gather")

    def batch(self, indices: torch.Tensor):
        """(frame table, pixel positions, targets) of the dataset ``indices``."""
        F = int(indices.numel())
        table = self.frame_table(F)
        pixels = torch.empty((F * self.height * self.width, 3), dtype=torch.float32, device=self.device)
        targets = torch.empty((F * self.height * self.width,), dtype=torch.float32, device=self.device)
        self.fill(indices, table, pixels, targets)
        return table, pixels, targets

    def geometry(self, indices: torch.Tensor):
        """(ray_origins (F,W,3), ray_dirs (F,W,3), pose_world_to_probe (F,4,4)) of the dataset
        ``indices`` (device int64), one launch, no synchronisation."""
        F = int(indices.numel())
        if indices.dtype != torch.int64 or indices.device != self.device:
            raise ValueError("indices must be an int64 tensor on the dataset's device")
        origins = torch.empty((F, self.width, 3), dtype=torch.float32, device=self.device)
        dirs = torch.empty((F, self.width, 3), dtype=torch.float32, device=self.device)
        pose = torch.empty((F, 4, 4), dtype=torch.float32, device=self.device)
        _lib.check(_lib.call("us3d_frames_geometry", _ptr(self.records), self.n, _ptr(indices.contiguous()), F,
                             self.width, _ptr(self.ray_origins), _ptr(self.ray_dirs), _ptr(self.poses),
                             _ptr(origins), _ptr(dirs), _ptr(pose), _ptr(self.status), _stream()),
                   "us3d_frames_geometry")
        return origins, dirs, pose

    def camera(self, indices: torch.Tensor):
        """UltraGS camera fields of the dataset ``indices`` (device int64): (viewmatrix (F,4,4),
        projmatrix (F,4,4), camera_center (F,3), tanfovx (F,), tanfovy (F,)); device gathers, no
        synchronisation (an index outside the dataset is clamped and recorded for ``check``)."""
        if indices.dtype != torch.int64 or indices.device != self.device:
            raise ValueError("indices must be an int64 tensor on the dataset's device")
        bad = ((indices < 0) | (indices >= self.n)).any().to(torch.int32)
        torch.maximum(self.status, bad.reshape(1), out=self.status)
        i = indices.clamp(0, self.n - 1)
        return (self.viewmatrix.index_select(0, i), self.projmatrix.index_select(0, i),
                self.camera_center.index_select(0, i), self.tanfovx.index_select(0, i), self.tanfovy.index_select(0, i))

    def check(self) -> None:
        """Raises if any index given to ``fill`` was out of range (synchronises)."""
        if int(self.status.item()):
            raise IndexError("a frame index outside the dataset was given")
