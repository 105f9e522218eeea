"""Drop-in UltraGray scanline B-mode renderer on B200 (same public names as the reference
package ops/ultragray_renderer/ultragray_renderer/__init__.py)."""

from .api import UltragrayRenderer
from .types import ProbeGeometry, UltragrayRenderConfig

__all__ = ["UltragrayRenderer", "UltragrayRenderConfig", "ProbeGeometry"]
