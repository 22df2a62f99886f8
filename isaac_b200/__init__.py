"""B200-native ISAAC in-situ rendering hot path.

``IsaacVisualization`` mirrors the reference's host object; the work runs in
hand-written sm_100a CUDA kernels behind the C ABI ``include/isaac_b200.h``
(library ``isaac_b200/_build/libisaac_b200.so``, built by ``isaac_b200.build``).
"""

from .visualization import (
    DefaultController,
    IsaacVisualization,
    ParticleSource,
    VolumeSource,
    modelview,
    perspective,
)

__all__ = [
    "DefaultController",
    "IsaacVisualization",
    "ParticleSource",
    "VolumeSource",
    "modelview",
    "perspective",
]
