"""Dark/flat-field correction, -log and the [A,V,U] -> [A,U,V] transpose in
one kernel (dgc_preprocess) against the same formula in FP64 numpy."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def reference(raw, dark, flat, layout, min_ratio):
    r = raw.astype(np.float64)
    d = 0.0 if dark is None else dark.astype(np.float64)
    f = 1.0 if flat is None else flat.astype(np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        ratio = (r - d) / (f - d)
    ratio = np.where(ratio >= min_ratio, ratio, min_ratio)  # NaN -> min_ratio
    p = -np.log(ratio)
    return p.transpose(0, 2, 1) if layout == "AVU" else p


@pytest.mark.parametrize("layout", ["AVU", "AUV"])
@pytest.mark.parametrize("A,U,V", [(3, 70, 45), (1, 32, 32), (5, 1, 67)])
def test_preprocess_matches_formula(layout, A, U, V):
    from dgc_b200.preprocessing import preprocess

    rng = np.random.default_rng(A * 100 + U + V)
    shape = (A, V, U) if layout == "AVU" else (A, U, V)
    dark = rng.uniform(90, 110, shape[1:]).astype(np.float32)
    flat = (dark + rng.uniform(3e4, 5e4, shape[1:])).astype(np.float32)
    raw = (dark + (flat - dark) * np.exp(-rng.uniform(0, 6, shape))).astype(np.float32)
    raw[0, 0, 0] = dark[0, 0] - 5.0          # below dark: clamped
    raw[-1, -1, -1] = dark[-1, -1]           # zero signal: clamped
    for d, f in ((dark, flat), (None, flat), (None, None)):
        out = preprocess(torch.tensor(raw, device="cuda"),
                         None if d is None else torch.tensor(d, device="cuda"),
                         None if f is None else torch.tensor(f, device="cuda"),
                         layout=layout, min_ratio=1e-6)
        want = reference(raw, d, f, layout, 1e-6)
        assert out.shape == (A, U, V)
        np.testing.assert_allclose(out.cpu().numpy(), want, rtol=2e-6, atol=2e-6)


def test_preprocess_feeds_the_operators():
    """A projection stored [A,V,U] as intensities comes back as the line
    integrals project() made (I0 = 1e4, no noise)."""
    import math

    import cbct_backprojector as cb
    from dgc_b200.phantoms import circular_geometry, ellipsoid_phantom
    from dgc_b200.preprocessing import preprocess

    vol = ellipsoid_phantom((32, 32, 32), seed=3, device="cuda", axis_range=(2.0, 8.0))
    geom = circular_geometry(6, 40, 36, 200.0, 120.0, 1.0, device="cuda")
    p = cb.project(vol, *geom, 1.0, 40, 36, step_size=0.5, voxel_size=1.0)
    intensity_avu = (1e4 * torch.exp(-p)).permute(0, 2, 1).contiguous()
    flat = torch.full((36, 40), 1e4, device="cuda")
    back = preprocess(intensity_avu, None, flat, layout="AVU")
    assert float((back - p).abs().max()) < 1e-5 * max(1.0, float(p.abs().max()))
    assert math.isfinite(float(back.sum()))
