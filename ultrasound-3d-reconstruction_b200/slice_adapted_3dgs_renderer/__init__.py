"""Drop-in slice-adapted 3DGS additive splatting on B200 (same public names as the
reference package ops/slice_adapted_3dgs_renderer/slice_adapted_3dgs_renderer/__init__.py)."""

from .api import additive_splat, additive_splat_bounded
from .fused import render_slice_adapted_3dgs

__all__ = ["additive_splat", "additive_splat_bounded", "render_slice_adapted_3dgs"]
