"""Module-name drop-in for the reference's native backprojector extension.

The reference's Python wrappers import ``src_cbct_backprojector_cuda`` by name
(TomSHINING/diff-geoCali ``cbct_backprojector/operator.py:20-29``) and call
``forward`` / ``backward`` with the signatures of
``csrc/src_cbct_backprojector_cuda.cu:524-543``.  With this directory on
``sys.path`` those calls run on libdgc's sm_100a kernels.
"""

from dgc_b200._ops import bp_backward as backward
from dgc_b200._ops import bp_forward as forward

__all__ = ["forward", "backward"]
