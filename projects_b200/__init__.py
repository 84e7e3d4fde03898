"""B200-native (sm_100a) gridrec: Fourier-gridding reconstruction of
parallel-beam tomography slices behind the reference's GridRec call surface.

Submodules: ``gridrec`` (C-ABI bindings, Plan, GridRec), ``phantom``
(seeded synthetic sinograms), ``build`` (in-tree nvcc build).
"""
from . import gridrec, phantom  # noqa: F401
from .gridrec import GridRec, Plan  # noqa: F401
