"""apirl_b200: B200-native Siddon projector / backprojector and MLEM/OSEM.

The compute path is the CUDA library apirl_b200/_build/libapirl_b200.so,
reached through its C ABI (include/apirl_b200.h).
"""
from .geometry import ImageGeom, Sino2DGeom, Sino3DGeom, subset_nproj  # noqa: F401
from ._lib import ApirlError, load as load_library  # noqa: F401
from .projector import (SiddonProjector, inverse_divide, add_bins, likelihood, mlem_threshold,  # noqa: F401
                        update_pixels, force_positive, osem_3d, mlem_3d, mlem_2d, set_iteration_hook)

__version__ = "0.1.0"
