"""Geometry calibration on the GPU: finite differences of the calibration loss
on 32 random views, convergence of the plain Adam loop, warm-start rejection."""

import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def setup_case(size=64, A=90, det=128, seed=5, I0=None):
    from dgc_b200 import calibration as C
    from dgc_b200.phantoms import circular_geometry, ellipsoid_phantom

    vol = ellipsoid_phantom((size,) * 3, seed=seed, device="cuda",
                            axis_range=(10 * size / 256, 80 * size / 256))
    nominal = circular_geometry(A, det, det, 1000.0, 600.0, 1.0, device="cuda")
    true = C.perturb_geometry(nominal, seed + 100)
    scan = C.ScanSetup(U=det, V=det)
    meas, mask = C.simulate_measurement(vol, true, scan, I0=I0, seed=seed)
    return C, vol, nominal, true, scan, meas, mask


def test_loss_gradient_finite_differences_on_32_views(oracle):
    """d/d(geometry) of MSE(project(vol, g), meas) against central differences.

    32 random (view, parameter) entries; the loss runs over rays whose trace
    (entry face, sample count, cells) is unchanged by the +-eps perturbation.
    The projector's ray set-up is FP32 (as the reference's): source position
    and direction are quantised at ~1e-4 mm, so the difference of each ray's
    projection carries that quantisation, and a per-view gradient is a sum of
    ray contributions that largely cancel.  The error bound is therefore
    relative to the summed magnitude of the ray contributions (the FP64
    oracle with FP64 ray set-up agrees with the analytic formula to 1e-8).
    """
    from dgc_b200 import _ops, project

    C, vol, nominal, true, scan, meas, _ = setup_case(size=48, A=64, det=96)

    def counts(g):
        return _ops.project_sample_counts(vol.shape, g, 1.0, scan.U, scan.V, 0.5, 1.0).cpu().numpy()

    # evaluate between nominal and truth, where the residual is not zero
    geom = [n + 0.7 * (t - n) for t, n in zip(true, nominal)]
    base = oracle.ray_traces(vol.shape, [g.cpu().numpy() for g in geom], 1.0, scan.U, scan.V,
                             0.5, 1.0, mode=1)
    base_counts = counts(geom)
    rng = np.random.default_rng(0)
    views = rng.choice(len(geom[0]), 32, replace=False)
    eps_by_family = [2e-4, 5e-2, 5e-2, 1e-2, 1e-2, 1e-2, 1e-2, 1e-2]
    checked = 0
    for i, a in enumerate(views):
        k = i % 8
        # halve the step until most of the view's rays keep their trace
        for eps in (eps_by_family[k] / 2**j for j in range(4)):
            plus = [g.clone() for g in geom]
            minus = [g.clone() for g in geom]
            plus[k][a] += eps
            minus[k][a] -= eps
            tp = oracle.ray_traces(vol.shape, [g.cpu().numpy() for g in plus], 1.0, scan.U,
                                   scan.V, 0.5, 1.0, mode=1)
            tm = oracle.ray_traces(vol.shape, [g.cpu().numpy() for g in minus], 1.0, scan.U,
                                   scan.V, 0.5, 1.0, mode=1)
            # the GPU's own sample counts guard the count exactly
            keep_np = ((base != 0) & (base == tp) & (base == tm) &
                       (counts(plus) == base_counts) & (counts(minus) == base_counts))
            if keep_np[a].mean() >= 0.5:
                break
        keep = torch.tensor(keep_np.astype(np.float32), device="cuda")
        if keep[a].mean() < 0.5:
            continue

        def proj(g):
            return project(vol, *g, 1.0, scan.U, scan.V, step_size=0.5).double()

        def loss(p):
            return ((p - meas.double()).square() * keep).sum() / keep.sum()

        gg = [g.clone().requires_grad_() for g in geom]
        analytic = torch.autograd.grad(loss(proj(gg)), gg[k])[0][a].item()
        with torch.no_grad():
            p0, pp, pm = proj(geom), proj(plus), proj(minus)
            h = (plus[k][a] - minus[k][a]).item()
            fd = ((loss(pp) - loss(pm)) / h).item()
            # summed magnitude of the per-ray contributions 2 (p - m) dp/dg
            scale = ((2 * (p0 - meas.double()) * (pp - pm) / h).abs() * keep).sum().item() / \
                keep.sum().item()
        assert abs(analytic - fd) <= 2e-2 * scale + 1e-7, (k, a, analytic, fd, scale)
        checked += 1
    assert checked >= 28


def test_plain_calibration_converges():
    C, vol, nominal, true, scan, meas, mask = setup_case(I0=1e5)
    res = C.calibrate(vol, meas, nominal, scan, iterations=150, true_geometry=true, mask=mask)
    first, last = res.history[0], res.history[-1]
    assert first["reproj_px"] > 1.0
    assert last["reproj_px"] < 0.25 * first["reproj_px"]
    assert res.final_loss < res.history[1]["loss"]


def test_warm_start_judge():
    C, vol, nominal, true, scan, meas, mask = setup_case()
    good = [t - n for t, n in zip(true, nominal)]
    bad = [torch.randn_like(n) * s for n, s in zip(nominal, (0.05, 20, 20, 8, 8, 5, 5, 5))]
    r_good = C.calibrate(vol, meas, nominal, scan, iterations=2, warm_start=good,
                         true_geometry=true, mask=mask)
    r_bad = C.calibrate(vol, meas, nominal, scan, iterations=2, warm_start=bad,
                        true_geometry=true, mask=mask)
    assert r_good.warm_start_accepted is True
    assert r_good.history[0]["reproj_px"] < 1e-3
    assert r_bad.warm_start_accepted is False
    # rejected prediction: the run starts from nominal
    assert abs(r_bad.history[0]["reproj_px"] - C.reprojection_error(
        nominal, true, C.lattice_points(vol.shape, device="cuda"), 1.0)) < 1e-9


def test_fused_step_matches_project_and_autograd():
    """dgc_project_mse_grad (one march) against project + masked MSE + autograd
    (two marches): the projection bitwise (the ray set-up is written with
    explicit fmaf / __fmul_rn, so both kernels march the same rays), the loss
    to 1e-5, the eight geometry gradients to 1e-5 (the upstream gradient
    2*scale*mask*(p - m) is rounded in a different order)."""
    from dgc_b200 import _ops, project

    C, vol, nominal, true, scan, meas, mask = setup_case(size=40, A=48, det=72, I0=1e5)
    geom = [n + 0.5 * (t - n) for t, n in zip(true, nominal)]
    for m in (mask, None):
        denom = float(meas.numel() if m is None else m.sum())
        loss, grads, proj = _ops.fp_mse_grad(vol, geom, 1.0, scan.U, scan.V, 0.5, 1.0, meas, m,
                                             1.0 / denom, return_projection=True)
        g = [x.clone().requires_grad_() for x in geom]
        p = project(vol, *g, 1.0, scan.U, scan.V, step_size=0.5, voxel_size=1.0)
        r = (p - meas).square()
        ref = (r if m is None else r * m).sum() / denom
        want = torch.autograd.grad(ref, g)
        torch.cuda.synchronize()
        assert torch.equal(proj, p.detach())
        assert math.isclose(float(loss.detach()), float(ref.detach()), rel_tol=1e-5)
        for k in range(8):
            a, b = grads[k].double(), want[k].double()
            assert float((a - b).norm() / b.norm()) < 1e-5, k


def test_fused_and_unfused_calibration_agree():
    C, vol, nominal, true, scan, meas, mask = setup_case(size=40, A=48, det=72, I0=1e5)
    pts = C.lattice_points(vol.shape, device="cuda")
    runs = [C.calibrate(vol, meas, nominal, scan, iterations=15, true_geometry=true, points=pts,
                        mask=mask, fused=f) for f in (True, False)]
    for a, b in zip(runs[0].history[1:], runs[1].history[1:]):
        assert math.isclose(a["loss"], b["loss"], rel_tol=1e-4)
    assert math.isclose(runs[0].history[-1]["reproj_px"], runs[1].history[-1]["reproj_px"],
                        rel_tol=1e-2)


def test_sharded_calibration_two_view_halves():
    """calibrate_sharded on two halves of the views, the sums over the
    halves standing in for the all-reduce: each half's offsets equal the
    whole calibration's bit for bit (the views' offsets are independent and
    the loss normalisation is the whole scan's)."""
    from dgc_b200 import calibration as C2
    from dgc_b200.sharded import view_shard

    C, vol, nominal, true, scan, meas, mask = setup_case(I0=1e5)
    whole = C.calibrate(vol, meas, nominal, scan, iterations=12, true_geometry=true, mask=mask)
    A = nominal[0].numel()
    halves = [view_shard(A, 2, r) for r in range(2)]
    for r, v in enumerate(halves):
        other = halves[1 - r]
        count_other = mask[other.start:other.stop].double().sum()
        calls = []

        def reduce(t, count_other=count_other, calls=calls):
            # without metrics or a warm start the first sum is the mask count;
            # the later ones (recorded losses) are not compared here
            calls.append(t.numel())
            return t + count_other if len(calls) == 1 else t

        sl = slice(v.start, v.stop)
        res = C2.calibrate(vol, meas[sl], [g[sl] for g in nominal], scan, iterations=12,
                           mask=mask[sl], reduce=reduce)
        for d, w in zip(res.delta, whole.delta):
            assert torch.equal(d.detach(), w.detach()[sl])
