"""lithobat_b200 — Lithobat's partially coherent imaging path on the NVIDIA B200.

Drop-in replacements for ``litho_sim.expose.compute_aerial_image`` and
``compute_aerial_planes``; the work runs in the sm_100a library
``liblitho_b200.so`` (C ABI in ``include/litho_b200.h``).
"""

from .aerial import (SOURCE_TILT_SIGN, LevelMasks, compute_aerial_batch, compute_aerial_image,
                     compute_aerial_planes, normalisation_scale)
from .config import GridConfig, OpticsConfig, ResistConfig
from .hopkins import SOCSKernels
from .source import Pole, Source, SourcePoints, build_source, source_points
from . import patterns
from . import torch_ops  # registers torch.ops.litho.*

__all__ = [
    "GridConfig", "LevelMasks", "OpticsConfig", "Pole", "SOCSKernels", "Source", "SourcePoints", "SOURCE_TILT_SIGN",
    "build_source", "compute_aerial_batch", "compute_aerial_image", "compute_aerial_planes",
    "normalisation_scale", "ResistConfig", "source_points",
]
