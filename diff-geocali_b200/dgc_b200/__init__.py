"""B200-native differentiable cone-beam CT operators (sm_100a): the implementation.

The public package ``cbct_backprojector`` (the drop-in for TomSHINING/diff-geoCali's
package of that name) re-exports this one.  The implementation carries its own
name so that the native-module shims (``src_cbct_*_cuda``) can load it while the
reference's own ``cbct_backprojector`` occupies that name on ``sys.path``.
All arithmetic runs in the in-tree CUDA library ``_lib/libdgc.so``.
"""

from .operator import backproject, detector_centers
from .filtering import fdk_filter, reconstruct_fdk
from .source_only_forward_projector import project, DifferentiableSourceOnlyForwardProjector

__all__ = [
    "backproject", "project", "DifferentiableSourceOnlyForwardProjector",
    "detector_centers", "fdk_filter", "reconstruct_fdk",
]
__version__ = "0.1.0"
