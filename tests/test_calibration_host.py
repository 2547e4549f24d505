"""Host-side calibration and warm-start logic on the CPU (pure torch): the
reprojection metric, the perturbation model, the network's output scales and
the autotuner-free parts of the warm-start module."""

import math

import torch


def nominal(A=12, U=64, V=48, px=1.0):
    from dgc_b200.phantoms import circular_geometry

    return circular_geometry(A, U, V, 1000.0, 600.0, px, device="cpu")


def test_reprojection_error_zero_and_detector_shift():
    from dgc_b200.calibration import lattice_points, reprojection_error

    g = nominal()
    pts = lattice_points((32, 32, 32), device="cpu")
    assert reprojection_error(g, g, pts, 1.0) == 0.0
    shifted = [t.clone() for t in g]
    shifted[3] = shifted[3] + 0.75   # det_u0 by 0.75 px moves every point by 0.75 px
    assert math.isclose(reprojection_error(g, shifted, pts, 1.0), 0.75, rel_tol=1e-9)
    both = [t.clone() for t in shifted]
    both[4] = both[4] - 1.0           # and det_v0 by 1 px: distance 1.25 px
    assert math.isclose(reprojection_error(g, both, pts, 1.0), 1.25, rel_tol=1e-9)


def test_detector_coordinates_match_the_backprojector_mapping():
    """A voxel at the isocentre lands on (u0, v0); one at height z lands
    z * sid / sod / pixel above it (bp.cu:48-72)."""
    from dgc_b200.calibration import detector_coordinates

    g = nominal(A=4, px=0.5)
    pts = torch.tensor([[0.0, 0.0, 0.0], [0.0, 0.0, 10.0]], dtype=torch.float64)
    d = detector_coordinates(pts, g, 0.5)
    torch.testing.assert_close(d[:, 0, 0].float(), g[3])
    torch.testing.assert_close(d[:, 0, 1].float(), g[4])
    torch.testing.assert_close((d[:, 1, 1] - d[:, 0, 1]).float(),
                               torch.full((4,), 10.0 * 1000.0 / 600.0 / 0.5))


def test_perturbation_model_is_seeded_and_sized():
    from dgc_b200.calibration import angle_error_deg, perturb_geometry

    g = nominal(A=2000)
    a = perturb_geometry(g, 3)
    b = perturb_geometry(g, 3)
    c = perturb_geometry(g, 4)
    assert all(torch.equal(x, y) for x, y in zip(a, b))
    assert not torch.equal(a[0], c[0])
    assert abs(angle_error_deg(a, g) - 0.3) < 0.03          # N(0, 0.3 deg)
    assert abs(float((a[5] - g[5]).std()) - 1.0) < 0.1       # src_x N(0, 1 mm)
    assert abs(float((a[3] - g[3]).std()) - 2.0) < 0.2       # det_u0 N(0, 2 px)
    assert abs(float((a[1] / g[1] - 1).std()) - 0.005) < 5e-4


def test_warm_start_scales_and_settings():
    from dgc_b200 import warmstart as WS

    s = WS.output_scales(WS.EVAL, device="cpu")
    assert s.shape == (8,)
    assert math.isclose(float(s[0]), math.radians(0.3), rel_tol=1e-6)
    assert math.isclose(float(s[3]), 2.0 / WS.EVAL.pixel)
    # the three acquisitions share the physical extent of the evaluation scan
    for acq in (WS.TRAIN, WS.HALF, WS.EVAL):
        assert math.isclose(acq.volume * acq.voxel, 512.0)
        assert math.isclose(acq.detector * acq.pixel, 768.0)
    assert WS.WARM_STAGES >= 1 and WS.WARM_CALIBRATION["warmup_iterations"] > 0


def test_committed_weights_load_on_cpu():
    from dgc_b200 import warmstart as WS

    ck = torch.load(WS.default_checkpoint(), map_location="cpu", weights_only=False)
    net = WS.WarmStartNet()
    net.load_state_dict(ck["state"])
    n = sum(p.numel() for p in net.parameters())
    assert 1.2e6 < n < 2.5e6
    assert ck["meta"]["steps"] >= 20000
    assert all(torch.isfinite(p).all() for p in net.parameters())
