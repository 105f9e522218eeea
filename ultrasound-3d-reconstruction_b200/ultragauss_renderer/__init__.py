"""Drop-in UltraGauss renderer (probe-plane 3D Mahalanobis slice splatting) on B200.

Same public names as the reference package ``ultragauss_renderer``
(ops/ultragauss_renderer/ultragauss_renderer/__init__.py:1-4).
"""

from .api import UltraGaussRenderer
from .types import SliceGeometry, UltraGaussRenderConfig

__all__ = ["UltraGaussRenderer", "SliceGeometry", "UltraGaussRenderConfig"]
