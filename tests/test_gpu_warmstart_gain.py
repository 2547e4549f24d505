"""What the trained warm-start network gains over calibration without it.

On held-out stacks of the training acquisition (seeds outside the training
range) the network's predicted geometry must land closer to the true
geometry than the nominal start (RMS reprojection distance), and a short
gradient calibration started from the prediction must end closer than the
same calibration started from nominal.  Uses the committed weights
(``cbct_backprojector/warmstart_weights.pt``), trained by
``warmstart.train`` on projector-generated stacks.
"""

import pytest

pytestmark = pytest.mark.gpu

HELD_OUT = (7, 11, 23, 42, 77, 101)


@pytest.fixture(scope="module")
def net():
    from dgc_b200 import warmstart as WS

    path = WS.default_checkpoint()
    assert path.exists(), f"trained weights missing: {path}"
    net, meta = WS.load(path)
    net.eval()
    return net


def test_prediction_beats_nominal(net):
    from dgc_b200 import warmstart as WS
    from dgc_b200.calibration import lattice_points

    acq = WS.TRAIN
    pts = lattice_points((acq.volume,) * 3, acq.voxel, device="cuda")
    nominal_mm, nn_mm = [], []
    for seed in HELD_OUT:
        st = WS.make_stack(acq, seed)
        delta = WS.predict(net, st["measured"], st["nominal_projection"], st["mask"],
                           st["nominal"], acq)
        pred = [n + d for n, d in zip(st["nominal"], delta)]
        nominal_mm.append(float(WS.reprojection_loss(st["nominal"], st["true"], pts, acq.pixel)))
        nn_mm.append(float(WS.reprojection_loss(pred, st["true"], pts, acq.pixel)))
    nominal_rms = (sum(nominal_mm) / len(nominal_mm)) ** 0.5
    nn_rms = (sum(nn_mm) / len(nn_mm)) ** 0.5
    assert nn_rms < 0.6 * nominal_rms, (nn_rms, nominal_rms)


def test_warm_started_calibration_reaches_target_faster(net):
    """From the network's multi-stage start with its calibration settings, the
    0.1 px target comes in fewer than half the iterations of calibration from
    nominal (46-52 vs 7-12 on held-out stacks when the settings were chosen)."""
    from dgc_b200 import warmstart as WS
    from dgc_b200.calibration import calibrate, lattice_points

    acq = WS.TRAIN
    st = WS.make_stack(acq, 42)
    pts = lattice_points(st["volume"].shape, acq.voxel, device="cuda")
    kw = dict(iterations=120, true_geometry=st["true"], points=pts, mask=st["mask"],
              target_px=0.1, stop_at_target=True)
    plain = calibrate(st["volume"], st["measured"], st["nominal"], acq.scan, **kw)
    warm = WS.predict(net, st["measured"], st["nominal_projection"], st["mask"], st["nominal"],
                      acq, volume=st["volume"], stages=WS.WARM_STAGES)
    nn = calibrate(st["volume"], st["measured"], st["nominal"], acq.scan, warm_start=warm,
                   **dict(kw, **WS.WARM_CALIBRATION))
    assert nn.warm_start_accepted
    assert nn.history[0]["reproj_px"] < 0.3 * plain.history[0]["reproj_px"]
    assert plain.iterations_to_target is not None and nn.iterations_to_target is not None
    assert 2 * nn.iterations_to_target < plain.iterations_to_target, (
        nn.iterations_to_target, plain.iterations_to_target)
