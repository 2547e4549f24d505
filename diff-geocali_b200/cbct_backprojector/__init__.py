"""B200-native differentiable cone-beam CT operators (sm_100a).

Drop-in for the ``cbct_backprojector`` package of TomSHINING/diff-geoCali: the
same public names, arguments, layouts ([D,H,W] volumes, [A,U,V] projections,
eight per-view geometry tensors) and autograd behaviour.  All arithmetic runs
in the in-tree CUDA library ``_lib/libdgc.so``.
"""

from .operator import backproject, detector_centers
from .filtering import fdk_filter, reconstruct_fdk
from .source_only_forward_projector import project, DifferentiableSourceOnlyForwardProjector

__all__ = [
    "backproject", "project", "DifferentiableSourceOnlyForwardProjector",
    "detector_centers", "fdk_filter", "reconstruct_fdk",
]
__version__ = "0.1.0"
