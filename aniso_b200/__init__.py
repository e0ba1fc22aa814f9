"""aniso_b200: a B200 (sm_100a) tile-based Gaussian-splat rasterizer behind the C ABI of
include/aniso_b200.h, a drop-in for the reference's aniso::GpuRenderer.

The library libaniso_b200.so is loaded by the first call that needs it, which fails if it is
missing; there is no CPU path.
"""
from . import scenes  # noqa: F401  (pure numpy, no library needed)
from ._lib import AnisoError, LIB_PATH  # noqa: F401
from .renderer import (BatchOptions, BatchRenderer, GpuRenderer, RenderOptions, colmap_load, keys_of,  # noqa: F401
                       sort_projection)
