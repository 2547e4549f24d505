"""Full-size checks (256^3 volume, 360 views of 384^2, the FDK workload's
shape) through properties that hold at any size: the forward projector and
its volume gradient are exact transposes (dot-product test), a constant volume
projects to step x samples per ray, the backprojector and its projection
gradient are exact transposes, and FDK reconstructs the phantom it was given.
The small-size parity tests pin the values themselves against the oracle."""

import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

D, A, U, V = 256, 360, 384, 384
SID, SOD, PX, STEP = 1000.0, 600.0, 1.0, 0.5


def geometry():
    from cbct_backprojector import detector_centers

    ang = torch.arange(A, dtype=torch.float32, device="cuda") * (2 * math.pi / A)
    full = lambda x: torch.full((A,), float(x), dtype=torch.float32, device="cuda")  # noqa: E731
    u0, v0 = detector_centers(full(0.0), full(0.0), U, V, PX)
    return [ang, full(SID), full(SOD), u0, v0, full(0.3), full(-0.2), full(0.1)]


def dot(a, b):
    return float((a.double() * b.double()).sum())


def test_projector_adjoint_dot_product():
    """<P v, g> = <v, P^T g> with P^T the volume gradient."""
    from cbct_backprojector import project

    g = torch.Generator(device="cuda").manual_seed(1)
    vol = torch.rand((D, D, D), device="cuda", generator=g).requires_grad_()
    geom = geometry()
    p = project(vol, *geom, PX, U, V, step_size=STEP, voxel_size=1.0)
    # positive factors: no cancellation, so a misplaced weight shows at once
    up = torch.rand(p.shape, device="cuda", generator=g)
    (gv,) = torch.autograd.grad(p, [vol], grad_outputs=up)
    lhs, rhs = dot(p.detach(), up), dot(vol.detach(), gv)
    assert abs(lhs - rhs) <= 2e-5 * abs(lhs), (lhs, rhs)


def test_constant_volume_projects_to_the_sample_count():
    """A volume of ones: each ray's integral is exactly step x its FP32
    sample count (the trilinear interpolant of a constant is that constant)."""
    from dgc_b200 import _ops, project

    geom = geometry()
    p = project(torch.ones((D, D, D), device="cuda"), *geom, PX, U, V, step_size=STEP,
                voxel_size=1.0)
    counts = _ops.project_sample_counts((D, D, D), geom, PX, U, V, STEP, 1.0)
    torch.cuda.synchronize()
    assert torch.equal(p, counts.float() * STEP)
    assert int(counts.sum()) > 2.5e10


def test_backprojector_adjoint_dot_product():
    """<B q, w> = <q, B^T w> with B^T the projection gradient."""
    from cbct_backprojector import backproject

    g = torch.Generator(device="cuda").manual_seed(2)
    geom = geometry()
    q = torch.rand((A, U, V), device="cuda", generator=g).requires_grad_()
    vol = backproject(q, *geom, PX, (D, D, D), 1.0)
    w = torch.rand(vol.shape, device="cuda", generator=g)
    (gq,) = torch.autograd.grad(vol, [q], grad_outputs=w)
    lhs, rhs = dot(vol.detach(), w), dot(q.detach(), gq)
    assert abs(lhs - rhs) <= 2e-5 * abs(lhs), (lhs, rhs)


def test_fdk_reconstructs_the_phantom():
    """project -> reconstruct_fdk of an ellipsoid phantom at the workload's
    size: the reconstruction follows the phantom (FDK's cone-beam and
    sampling errors are far below the phantom's contrast)."""
    from cbct_backprojector import project, reconstruct_fdk
    from dgc_b200.phantoms import ellipsoid_phantom

    vol = ellipsoid_phantom((D, D, D), n=12, seed=3, device="cuda")
    geom = geometry()
    geom[5:] = [torch.zeros_like(geom[5]) for _ in range(3)]
    p = project(vol, *geom, PX, U, V, step_size=STEP, voxel_size=1.0)
    rec = reconstruct_fdk(p, *geom, PX, (D, D, D), 1.0)
    c = D // 2
    a, b = vol[c - 64:c + 64].double(), rec[c - 64:c + 64].double()  # central slab
    corr = float(((a - a.mean()) * (b - b.mean())).sum() /
                 ((a - a.mean()).norm() * (b - b.mean()).norm()))
    err = float((b - a).abs().mean()) / float(a.abs().mean())
    assert corr > 0.9 and err < 0.35, (corr, err)
    assert np.isfinite(rec.cpu().numpy()).all() and bool((rec >= 0).all())
