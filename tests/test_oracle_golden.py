"""Pin the FP64 C oracle to the reference's own CPU oracles (golden fixtures).

The fixtures in tests/golden/ were produced by tests/golden/make_golden.py from
the reference's examples/check_operator.py, examples/check_forward_operator.py
and cbct_backprojector/filtering.py.  The oracle must reproduce their values
and their autograd gradients (which also validates the reference CUDA
kernels' analytic gradient formulas, restated by the oracle).
"""

import math

import numpy as np
import pytest

from conftest import GEOM_NAMES, golden_geometry, rel_l2


def test_backprojector_check_case(golden, oracle):
    d = golden("bp_check_case.npz")
    geom = golden_geometry(d)
    shape = tuple(int(s) for s in d["volume_shape"])
    off = tuple(d["volume_offset"])
    out = oracle.backproject(d["in_data"], geom, float(d["pixel_size"]), shape,
                             float(d["voxel_size"]), off)
    np.testing.assert_allclose(out, d["output"], rtol=1e-12, atol=1e-12)
    # the reference's independent scalar (math.fsum) evaluation of sum(out * upstream)
    assert math.isclose(float((out * d["upstream"]).sum()), float(d["scalar_loss"]),
                        rel_tol=1e-12, abs_tol=1e-12)
    gp, gg = oracle.backproject_backward(d["upstream"], d["in_data"], geom,
                                         float(d["pixel_size"]), float(d["voxel_size"]), off)
    np.testing.assert_allclose(gp, d["grad_data"], rtol=1e-10, atol=1e-12)
    for k, name in enumerate(GEOM_NAMES):
        np.testing.assert_allclose(gg[k], d["grad_" + name], rtol=1e-10, atol=1e-12,
                                   err_msg=name)


def test_forward_check_case(golden, oracle):
    d = golden("fp_check_case.npz")
    geom = golden_geometry(d)
    U, V = (int(x) for x in d["detector"])
    kw = dict(pixel_size=float(d["pixel_size"]), step_size=float(d["step_size"]),
              voxel_size=float(d["voxel_size"]))
    off = tuple(d["volume_offset"])
    out = oracle.project(d["in_data"], geom, kw["pixel_size"], U, V, kw["step_size"],
                         kw["voxel_size"], off, mode=0)
    np.testing.assert_allclose(out, d["output"], rtol=1e-12, atol=1e-12)
    counts = oracle.sample_counts(d["in_data"].shape, geom, kw["pixel_size"], U, V,
                                  kw["step_size"], kw["voxel_size"], off, mode=0)
    np.testing.assert_array_equal(counts, d["counts"])
    gv, gg = oracle.project_backward(d["upstream"], d["in_data"], geom, kw["pixel_size"],
                                     kw["step_size"], kw["voxel_size"], off, mode=0)
    np.testing.assert_allclose(gv, d["grad_data"], rtol=1e-10, atol=1e-12)
    for k, name in enumerate(GEOM_NAMES):
        np.testing.assert_allclose(gg[k], d["grad_" + name], rtol=1e-10, atol=1e-11,
                                   err_msg=name)


def test_forward_constant_zero_linear(golden, oracle):
    """check_forward_operator.py:158-173: constant, zero and linear volumes."""
    d = golden("fp_check_case.npz")
    geom = golden_geometry(d)
    U, V = (int(x) for x in d["detector"])
    args = (float(d["pixel_size"]), U, V, float(d["step_size"]), float(d["voxel_size"]),
            tuple(d["volume_offset"]))
    vol = d["in_data"]
    ones = oracle.project(np.ones_like(vol), geom, *args)
    np.testing.assert_allclose(ones, d["counts"] * float(d["step_size"]), rtol=1e-12, atol=1e-12)
    assert np.all(oracle.project(np.zeros_like(vol), geom, *args) == 0.0)
    other = vol[..., ::-1]
    lhs = oracle.project(1.3 * vol - 0.4 * other, geom, *args)
    rhs = 1.3 * oracle.project(vol, geom, *args) - 0.4 * oracle.project(other, geom, *args)
    np.testing.assert_allclose(lhs, rhs, rtol=1e-12, atol=1e-12)


def test_config1(golden, oracle):
    d = golden("fp_config1.npz")
    geom = golden_geometry(d)
    U, V = (int(x) for x in d["detector"])
    out = oracle.project(d["in_data"], geom, 1.0, U, V, 0.5, 1.0, mode=0)
    assert rel_l2(out, d["output"]) < 1e-13
    # the FP32 sample set of the CUDA kernels stays close to the closed-form rule
    assert rel_l2(oracle.project(d["in_data"], geom, 1.0, U, V, 0.5, 1.0, mode=1),
                  d["output"]) < 1e-5
    up = 2.0 * out / out.size  # d mean(p^2) / dp
    gv, gg = oracle.project_backward(up, d["in_data"], geom, 1.0, 0.5, 1.0, mode=0)
    assert rel_l2(gv, d["grad_data"]) < 1e-12
    for k, name in enumerate(GEOM_NAMES):
        assert rel_l2(gg[k], d["grad_" + name]) < 1e-12, name
    b = golden("bp_config1.npz")
    bgeom = golden_geometry(b)
    vol = oracle.backproject(b["in_data"], bgeom, 1.0, tuple(b["volume_shape"]), 1.0)
    assert rel_l2(vol, b["output"]) < 1e-13
    gp, gg = oracle.backproject_backward(b["upstream"], b["in_data"], bgeom, 1.0, 1.0)
    assert rel_l2(gp, b["grad_data"]) < 1e-12
    for k, name in enumerate(GEOM_NAMES):
        assert rel_l2(gg[k], b["grad_" + name]) < 1e-12, name


def test_fdk_filter(golden, oracle):
    """The Toeplitz restatement equals the reference's padded-FFT filter (fp32 outputs)."""
    d = golden("fdk_filter.npz")
    for i in range(int(d["n_cases"])):
        out = oracle.fdk_filter(d[f"c{i}_in"], float(d[f"c{i}_pixel"]), d[f"c{i}_sod"],
                                d[f"c{i}_sid"], float(d[f"c{i}_alpha"]))
        assert rel_l2(out, d[f"c{i}_out"]) < 2e-6, i


def test_fdk_taps_equal_fft_definition(oracle):
    """Taps restate filtering.py:87-103 (checked against numpy's FFT here)."""
    for U, px, alpha in [(9, 0.9, 0.8), (48, 1.0, 0.8), (17, 0.75, 1.0), (1, 1.0, 0.5)]:
        P = 1 << (2 * U - 1).bit_length()
        idx = np.arange(P)
        n = np.where(idx > P // 2, idx - P, idx)
        r = np.zeros(P)
        r[0] = 1.0 / (4 * px * px)
        odd = n % 2 != 0
        r[odd] = -1.0 / (np.pi * n[odd] * px) ** 2
        f = np.fft.fftfreq(P)
        hann = np.where(np.abs(f) <= alpha / 2, 0.5 + 0.5 * np.cos(2 * np.pi * f / alpha), 0.0)
        h = np.fft.ifft(np.fft.fft(r).real * hann).real[:U]
        np.testing.assert_allclose(oracle.fdk_taps(U, px, alpha), h, rtol=1e-10, atol=1e-14)


@pytest.mark.parametrize("mode", [0, 1])
def test_oracle_subset_matches_full(golden, oracle, mode):
    d = golden("fp_config1.npz")
    geom = golden_geometry(d)
    full = oracle.project(d["in_data"], geom, 1.0, 48, 40, 0.5, 1.0, mode=mode)
    rays = np.arange(0, full.size, 97)
    sub = oracle.project_rays(d["in_data"], geom, 1.0, 48, 40, 0.5, 1.0, rays, mode=mode)
    np.testing.assert_array_equal(sub, full.reshape(-1)[rays])


def test_fdk_filter_gradients_of_the_reference(golden, oracle):
    """The reference's autograd gradients of fdk_filter (golden) against the
    FP64 oracle: the projection gradient as the transpose of the linear
    filter (applied to every basis vector), the distance gradients by central
    differences -- the formulas the GPU backward implements."""
    d = golden("fdk_filter_grad.npz")
    for i in range(int(d["n_cases"])):
        p, up = d[f"c{i}_in"].astype(np.float64), d[f"c{i}_up"].astype(np.float64)
        px, alpha = float(d[f"c{i}_pixel"]), float(d[f"c{i}_alpha"])
        sod, sid = d[f"c{i}_sod"].astype(np.float64), d[f"c{i}_sid"].astype(np.float64)
        A, U, V = p.shape
        if A * U * V <= 600:  # transpose by basis vectors on the small cases
            gp = np.zeros_like(p)
            for idx in np.ndindex(*p.shape):
                e = np.zeros_like(p)
                e[idx] = 1.0
                gp[idx] = float((oracle.fdk_filter(e, px, sod, sid, alpha) * up).sum())
            assert rel_l2(d[f"c{i}_grad_in"], gp) < 1e-5, i
        for name, vec in (("sid", sid), ("sod", sod)):
            fd = np.zeros(A)
            for a in range(A):
                h = 1e-4 * vec[a]
                hi, lo = vec.copy(), vec.copy()
                hi[a] += h
                lo[a] -= h
                args = lambda v: (v, sid) if name == "sod" else (sod, v)  # noqa: E731
                yh = oracle.fdk_filter(p, px, *args(hi), alpha)
                yl = oracle.fdk_filter(p, px, *args(lo), alpha)
                fd[a] = float(((yh - yl) * up).sum()) / (2 * h)
            assert rel_l2(d[f"c{i}_grad_{name}"], fd) < 1e-4, (i, name)
