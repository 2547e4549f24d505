"""Original import path of the forward projector (reference ``source_only_forward_projector.py``)."""

from cbct_backprojector.source_only_forward_projector import (
    DifferentiableSourceOnlyForwardProjector,
    project,
)

__all__ = ["project", "DifferentiableSourceOnlyForwardProjector"]
