"""FDK on the GPU: the ramp filter against the reference's own fdk_filter
output (golden fixtures) and the FP64 oracle; reconstruct_fdk against the
reference pipeline (oracle filter -> reference CUDA backprojector -> pi/A,
clamp) and the FP64 oracle; an analytic-sphere sanity check.
"""

import math

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def cuda32(x):
    return torch.as_tensor(np.asarray(x), dtype=torch.float32).cuda()


def test_filter_against_reference_outputs(golden, oracle):
    from cbct_backprojector import fdk_filter

    d = golden("fdk_filter.npz")
    for i in range(int(d["n_cases"])):
        p = cuda32(d[f"c{i}_in"])
        sod, sid = d[f"c{i}_sod"], d[f"c{i}_sid"]
        scalar = np.all(sod == sod[0]) and np.all(sid == sid[0])
        out = fdk_filter(p, float(d[f"c{i}_pixel"]), float(sod[0]) if scalar else cuda32(sod),
                         float(sid[0]) if scalar else cuda32(sid), float(d[f"c{i}_alpha"]))
        assert out.is_contiguous() and out.shape == p.shape
        assert rel_l2(out.cpu(), d[f"c{i}_out"]) < 1e-5, i
        truth = oracle.fdk_filter(d[f"c{i}_in"], float(d[f"c{i}_pixel"]), sod, sid,
                                  float(d[f"c{i}_alpha"]))
        assert rel_l2(out.cpu(), truth) < 1e-5, i


def _circle_geometry(A, U, V, sid, sod, px):
    from cbct_backprojector import detector_centers

    angles = torch.arange(A, dtype=torch.float32, device="cuda") * (2 * math.pi / A)
    full = lambda x: torch.full((A,), float(x), dtype=torch.float32, device="cuda")  # noqa: E731
    u0, v0 = detector_centers(full(0.0), full(0.0), U, V, px)
    return [angles, full(sid), full(sod), u0, v0, full(0.0), full(0.0), full(0.0)]


@pytest.mark.parametrize("A,U,V,shape,alpha", [(36, 64, 48, (24, 32, 32), 0.8),
                                               (20, 37, 29, (17, 21, 19), 1.0)])
def test_reconstruct_matches_reference_pipeline(A, U, V, shape, alpha, ref_native, oracle):
    from cbct_backprojector import reconstruct_fdk

    _, ref_bp = ref_native
    rng = np.random.default_rng(A)
    proj = (rng.random((A, U, V)) * 4).astype(np.float32)
    geom = _circle_geometry(A, U, V, 300.0, 180.0, 1.0)
    off = (0.4, -0.3, 0.2)
    vol = reconstruct_fdk(cuda32(proj), *geom, 1.0, shape, 1.0, volume_offset=off, alpha=alpha)
    # reference pipeline: filter (FP64 oracle of filtering.py) -> reference CUDA
    # backprojection -> * pi/A -> clamp
    gnp = [g.cpu().numpy() for g in geom]
    filt = oracle.fdk_filter(proj, 1.0, gnp[2], gnp[1], alpha)
    ref = ref_bp.forward(cuda32(filt), *geom, 1.0, *shape, 1.0, *off)
    ref = (ref * (math.pi / A)).clamp_min(0.0)
    torch.cuda.synchronize()
    assert rel_l2(vol.cpu(), ref.cpu()) < 1e-5
    truth = oracle.reconstruct_fdk(proj, gnp, 1.0, shape, 1.0, off, alpha)
    assert rel_l2(vol.cpu(), truth) < 1e-5


def test_analytic_sphere():
    """examples/fdk.py's analytic sphere: the reconstruction is ~1 inside, ~0 outside."""
    from cbct_backprojector import reconstruct_fdk

    A, U, V, sid, sod, px, radius = 180, 128, 128, 1000.0, 500.0, 1.0, 10.0
    u = (torch.arange(U, dtype=torch.float32, device="cuda") - (U - 1) / 2) * px
    v = (torch.arange(V, dtype=torch.float32, device="cuda") - (V - 1) / 2) * px
    r2 = u[:, None].square() + v[None, :].square()
    d2 = sod**2 * r2 / (sid**2 + r2)
    view = 2.0 * torch.sqrt((radius**2 - d2).clamp_min(0.0))
    proj = view.unsqueeze(0).expand(A, -1, -1).contiguous()
    geom = _circle_geometry(A, U, V, sid, sod, px)
    vol = reconstruct_fdk(proj, *geom, px, (64, 64, 64), 0.5)
    centre = vol[24:40, 24:40, 24:40].mean().item()
    outside = vol[:, :4, :4].abs().mean().item()
    assert abs(centre - 1.0) < 0.05, centre
    assert outside < 0.05, outside
