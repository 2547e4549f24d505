"""Public drop-in package ``cbct_backprojector`` (B200, sm_100a).

The same public names, arguments, layouts ([D,H,W] volumes, [A,U,V]
projections, eight per-view geometry tensors) and autograd behaviour as the
``cbct_backprojector`` package of TomSHINING/diff-geoCali
(``cbct_backprojector/__init__.py:3-11``).

The implementation lives in the private package ``dgc_b200``.  This package
only names it: its three public submodules, ``operator``, ``filtering`` and
``source_only_forward_projector``, are the very module objects of
``dgc_b200`` (``cbct_backprojector.operator is dgc_b200.operator``), so code
written against either name shares one set of functions and autograd classes.
The native-module shims ``src_cbct_forwardprojector_cuda`` and
``src_cbct_backprojector_cuda`` import ``dgc_b200`` too, never this package,
so they also serve the reference's own ``cbct_backprojector`` when that one is
first on ``sys.path``.
"""

import sys as _sys

import dgc_b200 as _impl
from dgc_b200 import filtering, operator, source_only_forward_projector

for _module in (filtering, operator, source_only_forward_projector):
    _sys.modules[f"{__name__}.{_module.__name__.rsplit('.', 1)[1]}"] = _module

from dgc_b200 import (  # noqa: E402
    DifferentiableSourceOnlyForwardProjector,
    backproject,
    detector_centers,
    fdk_filter,
    project,
    reconstruct_fdk,
)

__all__ = [
    "backproject", "project", "DifferentiableSourceOnlyForwardProjector",
    "detector_centers", "fdk_filter", "reconstruct_fdk",
]
__version__ = _impl.__version__
