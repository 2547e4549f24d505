"""The public Python API rejects bad arguments with the reference's exception
types and messages (cbct_backprojector/operator.py:73-127,
source_only_forward_projector.py:30-71, filtering.py:16-179 of the
reference).  These checks run before any GPU work, so they run on CPU."""

import math

import pytest
import torch

import cbct_backprojector as cb
from cbct_backprojector.operator import _positive_scalar


def cpu_geom(A=3):
    return [torch.zeros(A) for _ in range(8)]


def test_package_surface():
    assert set(cb.__all__) == {"backproject", "project", "DifferentiableSourceOnlyForwardProjector",
                               "detector_centers", "fdk_filter", "reconstruct_fdk"}
    import source_only_forward_projector as legacy
    import src_cbct_backprojector_cuda as nbp
    import src_cbct_forwardprojector_cuda as nfp

    assert legacy.project is cb.project
    assert callable(nfp.forward) and callable(nfp.backward)
    assert callable(nbp.forward) and callable(nbp.backward)


def test_positive_scalar():
    assert _positive_scalar(2, "x") == 2.0
    with pytest.raises(TypeError):
        _positive_scalar(True, "x")
    with pytest.raises(TypeError):
        _positive_scalar("1", "x")
    with pytest.raises(ValueError):
        _positive_scalar(-1.0, "x")
    with pytest.raises(ValueError):
        _positive_scalar(math.inf, "x")


def test_detector_centers():
    assert cb.detector_centers(0.0, 0.0, 48, 40, 1.0) == (23.5, 19.5)
    assert cb.detector_centers(0.9, -1.8, 9, 7, 0.9) == (3.0, 5.0)
    du = torch.tensor([0.5], requires_grad=True)
    u0, _ = cb.detector_centers(du, 0.0, 10, 10, 0.5)
    u0.sum().backward()
    assert du.grad.item() == -2.0
    for bad in (1, 2.0, True):
        with pytest.raises(ValueError, match="detector_u must be an integer >= 2"):
            cb.detector_centers(0.0, 0.0, bad, 4, 1.0)
    with pytest.raises(TypeError):
        cb.detector_centers(0.0, 0.0, 4, 4, "1")


def test_project_validation():
    vol = torch.zeros(4, 4, 4)
    g = cpu_geom()
    with pytest.raises(TypeError, match="volume must be a torch.Tensor"):
        cb.project(vol.numpy(), *g, 1.0, 4, 4)
    with pytest.raises(ValueError, match="volume must be a CUDA float32 tensor"):
        cb.project(vol, *g, 1.0, 4, 4)
    with pytest.raises(ValueError, match="must be a CUDA float32 tensor"):
        cb.project(vol.double(), *g, 1.0, 4, 4)


def test_backproject_validation():
    proj = torch.zeros(3, 4, 4)
    g = cpu_geom()
    with pytest.raises(TypeError, match="projections must be a torch.Tensor"):
        cb.backproject(None, *g, 1.0, (2, 2, 2), 1.0)
    with pytest.raises(ValueError, match="projections must be a CUDA float32 tensor"):
        cb.backproject(proj, *g, 1.0, (2, 2, 2), 1.0)


def test_fdk_validation():
    with pytest.raises(TypeError, match="projections must be a torch.Tensor"):
        cb.fdk_filter([1.0], 1.0, 600.0, 1000.0)
    with pytest.raises(ValueError, match="nonempty"):
        cb.fdk_filter(torch.zeros(0, 4, 4), 1.0, 600.0, 1000.0)
    with pytest.raises(TypeError, match="dtype torch.float32"):
        cb.fdk_filter(torch.zeros(2, 4, 4, dtype=torch.float64), 1.0, 600.0, 1000.0)
    with pytest.raises(ValueError, match="alpha must satisfy"):
        cb.fdk_filter(torch.zeros(2, 4, 4), 1.0, 600.0, 1000.0, alpha=1.5)
    with pytest.raises(ValueError, match="sod must be a scalar or have one value per view"):
        cb.fdk_filter(torch.zeros(2, 4, 4), 1.0, [600.0, 600.0, 600.0], 1000.0)
    with pytest.raises(ValueError, match="sid must contain finite positive distances"):
        cb.fdk_filter(torch.zeros(2, 4, 4), 1.0, 600.0, -1.0)
    # the B200 build has no CPU path: a CPU tensor is refused, not silently filtered
    with pytest.raises(ValueError, match="requires CUDA"):
        cb.fdk_filter(torch.zeros(2, 4, 4), 1.0, 600.0, 1000.0)
    with pytest.raises(ValueError, match="reconstruct_fdk requires CUDA projections"):
        cb.reconstruct_fdk(torch.zeros(2, 4, 4), *cpu_geom(2), 1.0, (2, 2, 2), 1.0)
