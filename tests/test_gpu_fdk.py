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


@pytest.mark.parametrize("direction", [1.0, -1.0])
def test_short_scan_matches_oracle(direction, oracle):
    """reconstruct_fdk(short_scan=True): Parker weights (dgc_parker_weights)
    against the FP64 oracle's, and the weighted reconstruction against the
    oracle pipeline (weights x projections -> filter -> backprojection x view
    spacing -> clamp) at the parity bar."""
    from dgc_b200 import _ops, reconstruct_fdk

    A, U, V, px, sid, sod = 58, 48, 40, 1.0, 300.0, 180.0
    fan = math.atan(((U - 1) / 2 * px) / sid)
    span = math.pi + 2 * fan + 0.02
    angles = (0.4 + direction * np.linspace(0.0, span, A)).astype(np.float32)
    rng = np.random.default_rng(5)
    proj = (rng.random((A, U, V)) * 4).astype(np.float32)
    geom = [torch.tensor(angles, device="cuda")] + [
        torch.full((A,), x, dtype=torch.float32, device="cuda")
        for x in (sid, sod, (U - 1) / 2, (V - 1) / 2, 0.0, 0.0, 0.0)]
    w = _ops.parker_weights(geom[0], geom[1], U, px)
    w64 = oracle.parker_weights(angles, np.full(A, sid), U, px)
    assert float(np.abs(w.cpu().numpy() - w64).max()) < 1e-5
    shape, off = (20, 24, 24), (0.3, -0.2, 0.1)
    vol = reconstruct_fdk(cuda32(proj), *geom, px, shape, 1.0, volume_offset=off,
                          short_scan=True)
    gnp = [g.cpu().numpy().astype(np.float64) for g in geom]
    step = abs(float(angles[-1]) - float(angles[0])) / (A - 1)
    filt = oracle.fdk_filter(proj * w64[:, :, None], px, gnp[2], gnp[1], 0.8)
    truth = np.maximum(oracle.backproject(filt, gnp, px, shape, 1.0, off) * step, 0.0)
    assert rel_l2(vol.cpu(), truth) < 1e-5
    with pytest.raises(ValueError, match="short scan must cover"):
        reconstruct_fdk(cuda32(proj[:30]), *[g[:30] for g in geom], px, shape, 1.0,
                        short_scan=True)


def test_filter_gradients_match_the_reference(golden):
    """fdk_filter under autograd (dgc_fdk_filter_backward) against the
    reference's own autograd gradients (golden): projections, per-view sod and
    sid; and a scalar sid tensor receives the sum of the per-view gradients."""
    from cbct_backprojector import fdk_filter

    d = golden("fdk_filter_grad.npz")
    for i in range(int(d["n_cases"])):
        p = cuda32(d[f"c{i}_in"]).requires_grad_()
        sod = cuda32(d[f"c{i}_sod"]).requires_grad_()
        sid = cuda32(d[f"c{i}_sid"]).requires_grad_()
        up = cuda32(d[f"c{i}_up"])
        out = fdk_filter(p, float(d[f"c{i}_pixel"]), sod, sid, float(d[f"c{i}_alpha"]))
        assert rel_l2(out.detach().cpu(), d[f"c{i}_out"]) < 1e-5, i
        gp, gsod, gsid = torch.autograd.grad(out, [p, sod, sid], grad_outputs=up)
        assert rel_l2(gp.cpu(), d[f"c{i}_grad_in"]) < 1e-4, i
        assert rel_l2(gsod.cpu(), d[f"c{i}_grad_sod"]) < 1e-4, i
        assert rel_l2(gsid.cpu(), d[f"c{i}_grad_sid"]) < 1e-4, i
    # scalar distances: the gradient is the sum over views
    p = cuda32(d["c1_in"])
    sid_s = torch.tensor(float(d["c1_sid"][0]), device="cuda", requires_grad=True)
    sid_v = torch.full((p.shape[0],), float(d["c1_sid"][0]), device="cuda", requires_grad=True)
    up = cuda32(d["c1_up"])
    (g_s,) = torch.autograd.grad(fdk_filter(p, 1.0, 120.0, sid_s), [sid_s], grad_outputs=up)
    (g_v,) = torch.autograd.grad(fdk_filter(p, 1.0, 120.0, sid_v), [sid_v], grad_outputs=up)
    assert math.isclose(float(g_s), float(g_v.sum()), rel_tol=1e-5)
    # no grad needed: the plain filter, no autograd node
    assert fdk_filter(p, 1.0, 120.0, 180.0).grad_fn is None
