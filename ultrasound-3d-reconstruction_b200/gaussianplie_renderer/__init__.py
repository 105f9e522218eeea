"""Drop-in GaussianPile renderer (projected-slice us_focus splatting) on B200.

Same public names as the reference package (ops/gaussianplie_renderer/gaussianplie_renderer/
__init__.py:1-27).
"""

from .api import GaussianPlieRenderer
from .autograd import SHAPE_GRADIENTS, get_shape_gradients, set_shape_gradients
from .check import should_validate_inputs, validate_render_inputs
from .grid_geometry import build_slice_grid_pack
from .reference import build_covariance, focus_project, quat_to_matrix_wxyz, render_reference, world_to_camera
from .types import GaussianPlieRenderConfig

GAUSSIANPLIE_RENDERER_TAG = "gaussianplie_single_alpha_v2"

__all__ = [
    "GAUSSIANPLIE_RENDERER_TAG",
    "SHAPE_GRADIENTS",
    "get_shape_gradients",
    "set_shape_gradients",
    "GaussianPlieRenderer",
    "GaussianPlieRenderConfig",
    "build_covariance",
    "build_slice_grid_pack",
    "focus_project",
    "quat_to_matrix_wxyz",
    "render_reference",
    "should_validate_inputs",
    "validate_render_inputs",
    "world_to_camera",
]
