"""us3d_b200: B200-native (sm_100a) Gaussian rasterisation for freehand 3D ultrasound.

Host-side package over the C-ABI library ``lib/libus3d_b200.so``. The drop-in renderer
packages (``ultragauss_renderer`` and siblings) sit next to this package and keep the
call signatures of the reference project's renderers.
"""

from . import _lib
from .build import LIB_PATH, build

__all__ = ["LIB_PATH", "build", "_lib"]
