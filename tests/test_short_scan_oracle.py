"""Parker short-scan weights in the FP64 oracle (the restatement the GPU
kernel is checked against): the weights of every ray and its conjugate sum to
one, and a Parker-weighted short-scan FDK reconstruction of a phantom matches
the full-scan one in the central region, for scans turning either way."""

import math

import numpy as np
import pytest


@pytest.mark.parametrize("direction", [1.0, -1.0])
def test_conjugate_rays_sum_to_one(oracle, direction):
    U, px, sid = 65, 1.0, 200.0
    fan = math.atan(((U - 1) / 2 * px) / sid)
    span = math.pi + 2 * fan + 0.05
    # a dense scan so that conjugates fall on (nearly) sampled views
    A = 4001
    angles = 0.3 + direction * np.linspace(0.0, span, A)
    w = oracle.parker_weights(angles, np.full(A, sid), U, px)
    assert w.min() >= 0.0 and w.max() <= 1.0 + 1e-12
    uc = (np.arange(U) - (U - 1) / 2) * px
    gam = direction * np.arctan(uc / sid)  # the fan angle as the scan direction sees it
    beta = direction * (angles - angles[0])
    step = span / (A - 1)
    for u in (0, 10, 32, 50, 64):
        for b in np.linspace(0.0, math.pi, 23):
            a = int(round(b / step))
            bc = beta[a] + math.pi + 2 * gam[u]  # conjugate view of (beta, gamma)
            ac = int(round(bc / step))
            if ac >= A:
                continue
            uconj = U - 1 - u                     # -gamma
            total = w[a, u] + w[ac, uconj]
            assert abs(total - 1.0) < 5e-3, (u, b, total)


@pytest.mark.parametrize("direction", [1.0, -1.0])
def test_short_scan_reconstruction_matches_full_scan(oracle, direction):
    from dgc_b200.phantoms import ellipsoid_phantom

    N, U, V, px, sid, sod = 32, 64, 64, 1.0, 200.0, 120.0
    vol = ellipsoid_phantom((N, N, N), n=6, seed=2, device="cpu",
                            axis_range=(3.0, 10.0)).numpy().astype(np.float64)

    def geom(angles):
        A = len(angles)
        return [angles, np.full(A, sid), np.full(A, sod), np.full(A, (U - 1) / 2),
                np.full(A, (V - 1) / 2), np.zeros(A), np.zeros(A), np.zeros(A)]

    d = 2 * math.pi / 180
    full = np.arange(180) * d
    fan = math.atan(((U - 1) / 2 * px) / sid)
    ns = int(math.ceil((math.pi + 2 * fan) / d)) + 1
    short = direction * np.arange(ns) * d
    pf = oracle.project(vol, geom(full), px, U, V, 0.5, 1.0)
    ref = oracle.reconstruct_fdk(pf, geom(full), px, (N, N, N), 1.0)
    ps = oracle.project(vol, geom(short), px, U, V, 0.5, 1.0)
    w = oracle.parker_weights(short, np.full(ns, sid), U, px)
    g = geom(short)
    filt = oracle.fdk_filter(ps * w[:, :, None], px, g[2], g[1], 0.8)
    rec = np.maximum(oracle.backproject(filt, g, px, (N, N, N), 1.0) * d, 0.0)
    c = slice(8, 24)
    err = np.linalg.norm((rec - ref)[c, c, c]) / np.linalg.norm(ref[c, c, c])
    unweighted = np.maximum(oracle.backproject(oracle.fdk_filter(ps, px, g[2], g[1], 0.8), g, px,
                                               (N, N, N), 1.0) * d / 2, 0.0)
    err_unweighted = (np.linalg.norm((unweighted - ref)[c, c, c]) /
                      np.linalg.norm(ref[c, c, c]))
    assert err < 0.06 and err < 0.25 * err_unweighted, (err, err_unweighted)
