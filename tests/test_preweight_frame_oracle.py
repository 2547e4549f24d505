"""The offset-aware cosine preweight on the CPU: the FP64 oracle's frame
restatement against the pinned centred filter (a centred frame reproduces it
bit for bit), the frame against the projector's own source and detector points
(the weight is the cosine of each ray's angle to the detector normal), the
torch ``preweight_frame`` against the oracle's, Parker weights in a frame,
``fdk_filter``'s frame argument checks, and the oracle's analytic filter
gradients (the adjoint's formulas) against its own finite differences."""

import math

import numpy as np
import pytest
import torch


def _geometry(A, U, V, seed, px):
    rng = np.random.default_rng(seed)
    return np.stack([
        rng.uniform(0, 2 * np.pi, A), 300 + rng.normal(0, 3, A), 180 + rng.normal(0, 2, A),
        (U - 1) / 2 + rng.normal(0, 2, A), (V - 1) / 2 + rng.normal(0, 2, A),
        rng.normal(0, 1.5, A), rng.normal(0, 1.5, A), rng.normal(0, 1.5, A)])


def test_centred_frame_is_the_pinned_filter(oracle):
    A, U, V = 3, 21, 14
    rng = np.random.default_rng(1)
    p = rng.random((A, U, V))
    sod, sid = 180 + rng.normal(0, 2, A), 300 + rng.normal(0, 3, A)
    plain = oracle.fdk_filter(p, 0.9, sod, sid, 0.8)
    framed = oracle.fdk_filter(p, 0.9, sod, sid, 0.8, frame=(sid, (U - 1) / 2, (V - 1) / 2))
    assert np.array_equal(plain, framed)
    # each entry alone falls back to its centred default
    assert np.array_equal(plain, oracle.fdk_filter(p, 0.9, sod, sid, 0.8, (None, None, None)))


def test_frame_weight_is_the_ray_cosine(oracle):
    """An impulse at pixel (k, j) of view a filters to h[0] * w * px * sid/sod
    at that pixel, so the oracle's weight w in the frame of
    ``oracle.preweight_frame`` must be the cosine between the ray from the
    source to the detector point of (k, j) and the detector normal, with the
    source and detector points of the projector (fp.cu:115-170)."""
    A, U, V, px = 6, 33, 27, 0.7
    g = _geometry(A, U, V, 2, px)
    rng = np.random.default_rng(3)
    ks, js = rng.integers(0, U, A), rng.integers(0, V, A)
    p = np.zeros((A, U, V))
    p[np.arange(A), ks, js] = 1.0
    out = oracle.fdk_filter(p, px, g[2], g[1], 0.8, frame=oracle.preweight_frame(g, px))
    h0 = oracle.fdk_taps(U, px, 0.8)[0]
    for a in range(A):
        b, sid, sod, u0, v0, sx, sy, sz = g[:, a]
        c, s = math.cos(b), math.sin(b)
        src = np.array([-sod * s + sx, sod * c + sy, sz])
        up, vp = (ks[a] - u0) * px, (js[a] - v0) * px
        det = np.array([up * c - (sod - sid) * s, up * s + (sod - sid) * c, vp])
        ray = det - src
        normal = np.array([-s, c, 0.0])
        cosine = abs(ray @ normal) / np.linalg.norm(ray)
        w = out[a, ks[a], js[a]] / (h0 * px * sid / sod)
        assert math.isclose(w, cosine, rel_tol=1e-12), (a, w, cosine)


def test_frame_foot_is_perpendicular(oracle):
    """The frame's centre is the foot of the perpendicular from the source and
    its distance the source's distance to the detector plane; the torch
    ``preweight_frame`` agrees with the oracle's."""
    from dgc_b200.filtering import preweight_frame

    A, U, V, px = 9, 40, 30, 1.3
    g = _geometry(A, U, V, 4, px)
    dist, fu, fv = oracle.preweight_frame(g, px)
    for a in range(A):
        b, sid, sod, u0, v0, sx, sy, sz = g[:, a]
        c, s = math.cos(b), math.sin(b)
        src = np.array([-sod * s + sx, sod * c + sy, sz])
        up, vp = (fu[a] - u0) * px, (fv[a] - v0) * px
        foot = np.array([up * c - (sod - sid) * s, up * s + (sod - sid) * c, vp])
        ray = foot - src
        normal = np.array([-s, c, 0.0])
        assert np.linalg.norm(np.cross(ray, normal)) < 1e-9 * np.linalg.norm(ray)
        assert math.isclose(np.linalg.norm(ray), dist[a], rel_tol=1e-12)
    t = preweight_frame(*[torch.tensor(x) for x in g], px)
    for mine, ref in zip(t, (dist, fu, fv)):
        assert np.allclose(mine.numpy(), ref, rtol=0, atol=1e-10)
    # no offsets, centred detector: the reference's centred weight
    z = g.copy()
    z[3], z[4], z[5:] = (U - 1) / 2, (V - 1) / 2, 0.0
    dist0, fu0, fv0 = oracle.preweight_frame(z, px)
    assert np.array_equal(dist0, z[1]) and np.all(fu0 == (U - 1) / 2) and np.all(fv0 == (V - 1) / 2)


def test_parker_weights_in_a_frame(oracle):
    A, U, px, sid = 40, 31, 1.0, 300.0
    fan = math.atan(((U - 1) / 2 + 4) * px / (sid - 5))
    angles = np.linspace(0.0, math.pi + 2 * fan + 0.01, A)
    base = oracle.parker_weights(angles, np.full(A, sid), U, px)
    same = oracle.parker_weights(angles, np.full(A, sid), U, px, np.full(A, sid),
                                 np.full(A, (U - 1) / 2))
    assert np.array_equal(base, same)
    # a frame shifted by s columns is the centred table of a detector shifted the same way
    shifted = oracle.parker_weights(angles, np.full(A, sid), U, px, np.full(A, sid - 5.0),
                                    np.full(A, (U - 1) / 2 + 4))
    gam = np.arctan((np.arange(U) - ((U - 1) / 2 + 4)) * px / (sid - 5.0))
    beta = angles[:, None]
    gmax = 0.5 * (angles[-1] - angles[0] - math.pi)
    inner = (beta >= 2 * (gmax - gam)) & (beta <= math.pi - 2 * gam)
    assert np.all(shifted[inner] == 1.0)
    # every ray and its conjugate weigh 1 together (sampled where the conjugate lands inside)
    for a in range(0, A, 5):
        for u in range(U):
            bc = angles[a] + math.pi + 2 * gam[u]
            if bc > angles[-1] or not gmax > abs(gam[u]):
                continue
            gc = -gam[u]
            rise = (bc < 2 * (gmax - gc))
            w_c = (math.sin(0.25 * math.pi * bc / (gmax - gc)) ** 2 if rise else
                   1.0 if bc <= math.pi - 2 * gc else
                   math.sin(0.25 * math.pi * (math.pi + 2 * gmax - bc) / (gmax + gc)) ** 2)
            assert math.isclose(shifted[a, u] + w_c, 1.0, abs_tol=1e-9)


def test_fdk_filter_frame_argument_checks():
    from cbct_backprojector import fdk_filter

    p = torch.zeros(3, 8, 6)
    with pytest.raises(TypeError, match="frame must be"):
        fdk_filter(p, 1.0, 180.0, 300.0, frame=(1.0, 2.0))
    with pytest.raises(ValueError, match="frame dist"):
        fdk_filter(p, 1.0, 180.0, 300.0, frame=(-1.0, None, None))
    with pytest.raises(ValueError, match="frame u"):
        fdk_filter(p, 1.0, 180.0, 300.0, frame=(None, float("nan"), None))
    with pytest.raises(ValueError, match="one value per view"):
        fdk_filter(p, 1.0, 180.0, 300.0, frame=(None, None, torch.zeros(2)))
    with pytest.raises(ValueError, match="CUDA"):
        fdk_filter(p, 1.0, 180.0, 300.0, frame=(300.0, 3.5, 2.5))


@pytest.mark.parametrize("framed", [False, True])
def test_filter_gradient_restatement(oracle, framed):
    """The oracle's analytic filter gradients (the formulas the CUDA adjoint
    evaluates) against central differences of the oracle filter, per view,
    with and without a preweight frame; the projection gradient by the
    dot-product identity <grad_P, Q> = <g, F(Q)>."""
    A, U, V, px, alpha = 3, 17, 11, 0.9, 0.85
    rng = np.random.default_rng(21)
    p = rng.random((A, U, V))
    g = rng.standard_normal((A, U, V))
    sod, sid = 180 + rng.normal(0, 2, A), 300 + rng.normal(0, 3, A)
    frame = ([sid + rng.normal(0, 4, A), (U - 1) / 2 + rng.normal(0, 2, A),
              (V - 1) / 2 + rng.normal(0, 2, A)] if framed else None)
    grads = oracle.fdk_filter_backward(g, p, px, sod, sid, alpha, frame)
    names = ["sod", "sid"] + (["dist", "u", "v"] if framed else [])
    assert sorted(grads) == sorted(names + ["P"])
    base = [sod, sid] + (list(frame) if framed else [])

    def loss(vals):
        fr = vals[2:] if framed else None
        return float((g * oracle.fdk_filter(p, px, vals[0], vals[1], alpha, fr)).sum())

    for k, name in enumerate(names):
        h = 1e-4 * (100.0 if k < 3 else 1.0)
        for a in range(A):
            plus = [b.copy() for b in base]
            minus = [b.copy() for b in base]
            plus[k][a] += h
            minus[k][a] -= h
            fd = (loss(plus) - loss(minus)) / (2 * h)
            assert math.isclose(grads[name][a], fd, rel_tol=1e-6, abs_tol=1e-9), (name, a)
    q = rng.standard_normal((A, U, V))
    lhs = float((grads["P"] * q).sum())
    rhs = float((g * oracle.fdk_filter(q, px, sod, sid, alpha, frame)).sum())
    assert math.isclose(lhs, rhs, rel_tol=1e-12)


def test_preweight_frame_gradients_reach_the_geometry():
    """preweight_frame is torch arithmetic, so autograd carries frame
    gradients into the geometry: d(dist)/d(sid) = 1, d(u)/d(det_u0) = 1,
    d(u)/d(src_x) = cos(b)/px, d(dist)/d(src_x) = -sin(b), d(v)/d(src_z) = 1/px,
    and d(u)/d(angle) = (-sx sin b + sy cos b)/px; sod does not enter."""
    from dgc_b200.filtering import preweight_frame

    A, px = 5, 0.8
    g = [torch.tensor(x, requires_grad=True) for x in _geometry(A, 16, 12, 9, px)]
    dist, u, v = preweight_frame(*g, px)
    b, sx, sy = (t.detach() for t in (g[0], g[5], g[6]))
    gd = torch.autograd.grad(dist.sum(), g, allow_unused=True, retain_graph=True)
    gu = torch.autograd.grad(u.sum(), g, allow_unused=True, retain_graph=True)
    gv = torch.autograd.grad(v.sum(), g, allow_unused=True)
    assert torch.allclose(gd[1], torch.ones(A, dtype=torch.float64))
    assert torch.allclose(gd[5], -torch.sin(b)) and torch.allclose(gd[6], torch.cos(b))
    assert torch.allclose(gu[3], torch.ones(A, dtype=torch.float64))
    assert torch.allclose(gu[5], torch.cos(b) / px) and torch.allclose(gu[6], torch.sin(b) / px)
    assert torch.allclose(gu[0], (-sx * torch.sin(b) + sy * torch.cos(b)) / px)
    assert torch.allclose(gv[4], torch.ones(A, dtype=torch.float64))
    assert torch.allclose(gv[7], torch.full((A,), 1 / px, dtype=torch.float64))
    assert gd[2] is None and gu[2] is None and gv[2] is None  # sod
