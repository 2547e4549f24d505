"""Module-name drop-in for the reference's native forward-projector extension.

The reference's Python wrappers import ``src_cbct_forwardprojector_cuda`` by
name (TomSHINING/diff-geoCali ``cbct_backprojector/source_only_forward_projector.py:17-27``)
and call ``forward`` / ``backward`` with the signatures of
``csrc/src_cbct_forwardprojector_cuda.cu:732-758``.  With this directory on
``sys.path`` those calls run on libdgc's sm_100a kernels.
"""

from dgc_b200._ops import fp_backward as backward
from dgc_b200._ops import fp_forward as forward

__all__ = ["forward", "backward"]
