"""The offset-aware cosine preweight on the GPU (dgc_fdk_filter_ex,
dgc_fdk_filter_backward_ex, dgc_parker_weights_ex, dgc_reconstruct_fdk_ex)
against the FP64 oracle: the filter in a frame, its gradients (finite
differences of the oracle; the projection gradient by the dot-product test),
a centred frame reproducing the reference's filter and reconstruction bit for
bit, and full- and short-scan reconstructions with ``offset_preweight``."""

import math

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def cuda32(x):
    return torch.as_tensor(np.asarray(x), dtype=torch.float32).cuda()


def _case(A=5, U=40, V=28, seed=3):
    rng = np.random.default_rng(seed)
    p = (rng.random((A, U, V)) * 4).astype(np.float32)
    sod = (180 + rng.normal(0, 2, A)).astype(np.float32)
    sid = (300 + rng.normal(0, 3, A)).astype(np.float32)
    frame = [(sid + rng.normal(0, 4, A)).astype(np.float32),
             ((U - 1) / 2 + rng.normal(0, 3, A)).astype(np.float32),
             ((V - 1) / 2 + rng.normal(0, 2, A)).astype(np.float32)]
    return p, sod, sid, frame


def test_framed_filter_matches_oracle(oracle):
    from cbct_backprojector import fdk_filter

    p, sod, sid, frame = _case()
    px, alpha = 0.8, 0.9
    for pick in ((0, 1, 2), (1,), (0,), (2,), (1, 2)):
        fr = [frame[k] if k in pick else None for k in range(3)]
        out = fdk_filter(cuda32(p), px, cuda32(sod), cuda32(sid), alpha,
                         frame=[None if f is None else cuda32(f) for f in fr])
        truth = oracle.fdk_filter(p, px, sod, sid, alpha, frame=fr)
        assert rel_l2(out.cpu(), truth) < 1e-5, pick
    # scalars broadcast over the views
    out = fdk_filter(cuda32(p), px, cuda32(sod), cuda32(sid), alpha, frame=(310.0, 21.5, 12.0))
    truth = oracle.fdk_filter(p, px, sod, sid, alpha, frame=(310.0, 21.5, 12.0))
    assert rel_l2(out.cpu(), truth) < 1e-5


def test_centred_frame_is_the_reference_filter():
    from cbct_backprojector import fdk_filter

    p, sod, sid, _ = _case(seed=7)
    A, U, V = p.shape
    plain = fdk_filter(cuda32(p), 0.8, cuda32(sod), cuda32(sid))
    framed = fdk_filter(cuda32(p), 0.8, cuda32(sod), cuda32(sid),
                        frame=(cuda32(sid), torch.full((A,), (U - 1) / 2, device="cuda"),
                               torch.full((A,), (V - 1) / 2, device="cuda")))
    assert torch.equal(plain, framed)


def test_framed_filter_gradients(oracle):
    """Per-view gradients of L = sum(g * fdk_filter(P, frame)) for sod, sid
    and the frame's dist, u, v against central differences of the FP64 oracle;
    the projection gradient against the dot-product identity
    <grad_P, Q> = <g, F(Q)> with the oracle's F."""
    from cbct_backprojector import fdk_filter

    p, sod, sid, frame = _case(seed=11)
    A = p.shape[0]
    px, alpha = 0.8, 0.9
    g = np.random.default_rng(12).standard_normal(p.shape).astype(np.float32)
    ins = [cuda32(x).requires_grad_() for x in (p, sod, sid, *frame)]
    out = fdk_filter(ins[0], px, ins[1], ins[2], alpha, frame=ins[3:])
    grads = torch.autograd.grad(out, ins, grad_outputs=cuda32(g))

    base = [np.asarray(x, np.float64) for x in (sod, sid, *frame)]

    def loss(vals):
        y = oracle.fdk_filter(p, px, vals[0], vals[1], alpha, frame=vals[2:])
        return float((g.astype(np.float64) * y).sum())

    for k, name in enumerate(("sod", "sid", "dist", "u", "v")):
        h = 1e-3 if k >= 3 else 1e-2
        fd = np.empty(A)
        for a in range(A):
            plus = [b.copy() for b in base]
            minus = [b.copy() for b in base]
            plus[k][a] += h
            minus[k][a] -= h
            fd[a] = (loss(plus) - loss(minus)) / (2 * h)
        assert rel_l2(grads[k + 1].cpu(), fd) < 1e-4, (name, grads[k + 1].cpu().numpy(), fd)
    q = np.random.default_rng(13).standard_normal(p.shape)
    lhs = float((grads[0].cpu().numpy().astype(np.float64) * q).sum())
    rhs = float((g.astype(np.float64) *
                 oracle.fdk_filter(q, px, sod, sid, alpha, frame=frame)).sum())
    assert math.isclose(lhs, rhs, rel_tol=1e-5)
    # a frame entry without requires_grad gets no gradient and changes nothing else
    ins2 = [cuda32(x).requires_grad_() for x in (p, sod, sid)]
    out2 = fdk_filter(ins2[0], px, ins2[1], ins2[2], alpha,
                      frame=[cuda32(f) for f in frame])
    g2 = torch.autograd.grad(out2, ins2, grad_outputs=cuda32(g))
    for a_, b_ in zip(g2, grads[:3]):
        assert torch.equal(a_, b_)


def _offset_geometry(A, U, V, seed, angles=None):
    rng = np.random.default_rng(seed)
    if angles is None:
        angles = np.arange(A) * (2 * np.pi / A)
    cols = [angles, np.full(A, 300.0), np.full(A, 180.0), (U - 1) / 2 + rng.normal(0, 2, A),
            (V - 1) / 2 + rng.normal(0, 2, A), rng.normal(0, 1.5, A), rng.normal(0, 1.5, A),
            rng.normal(0, 1.5, A)]
    return [np.asarray(c, np.float32) for c in cols]


def test_offset_preweight_reconstruction(oracle):
    from cbct_backprojector import reconstruct_fdk

    A, U, V, shape, off, px = 36, 48, 40, (20, 24, 22), (0.4, -0.3, 0.2), 1.0
    geom = _offset_geometry(A, U, V, 5)
    proj = (np.random.default_rng(6).random((A, U, V)) * 4).astype(np.float32)
    vol = reconstruct_fdk(cuda32(proj), *map(cuda32, geom), px, shape, 1.0, volume_offset=off,
                          offset_preweight=True)
    truth = oracle.reconstruct_fdk(proj, geom, px, shape, 1.0, off, 0.8, offset_preweight=True)
    assert rel_l2(vol.cpu(), truth) < 1e-5
    plain = oracle.reconstruct_fdk(proj, geom, px, shape, 1.0, off, 0.8)
    assert rel_l2(plain, truth) > 1e-4  # the offsets do change the weights
    # centred detector, no source offsets: the reference's reconstruction, bit for bit
    c = [geom[0], geom[1], geom[2], np.full(A, (U - 1) / 2, np.float32),
         np.full(A, (V - 1) / 2, np.float32)] + [np.zeros(A, np.float32)] * 3
    a = reconstruct_fdk(cuda32(proj), *map(cuda32, c), px, shape, 1.0, offset_preweight=True)
    b = reconstruct_fdk(cuda32(proj), *map(cuda32, c), px, shape, 1.0)
    assert torch.equal(a, b)
    # a source offset that puts it behind the detector plane is refused
    behind = [x.copy() for x in c]
    behind[6][0] = -400.0  # src_y at angle 0: ds_n = -400 < -sid
    with pytest.raises(ValueError, match="in front of the detector plane"):
        reconstruct_fdk(cuda32(proj), *map(cuda32, behind), px, shape, 1.0,
                        offset_preweight=True)


def test_offset_preweight_short_scan(oracle):
    from dgc_b200 import _ops, reconstruct_fdk
    from dgc_b200.filtering import preweight_frame

    A, U, V, px, shape, off = 60, 48, 40, 1.0, (20, 24, 24), (0.3, -0.2, 0.1)
    probe = _offset_geometry(A, U, V, 8)  # the offsets; the angles below do not draw
    shift = np.abs(probe[5]) + np.abs(probe[6])  # bounds |ds_u| and |ds_n| at every angle
    reach = np.maximum(probe[3], U - 1 - probe[3]) * px + shift
    fan = float(np.max(np.arctan(reach / (probe[1] - shift))))
    angles = (0.3 + np.linspace(0.0, math.pi + 2 * fan + 0.02, A)).astype(np.float32)
    geom = _offset_geometry(A, U, V, 8, angles)
    g = [cuda32(x) for x in geom]
    frame = preweight_frame(*g, px)
    w = _ops.parker_weights(g[0], g[1], U, px, frame[0], frame[1])
    d64, u64, v64 = oracle.preweight_frame(geom, px)
    w64 = oracle.parker_weights(geom[0], geom[1], U, px, d64, u64)
    assert float(np.abs(w.cpu().numpy() - w64).max()) < 1e-5
    proj = (np.random.default_rng(9).random((A, U, V)) * 4).astype(np.float32)
    vol = reconstruct_fdk(cuda32(proj), *g, px, shape, 1.0, volume_offset=off, short_scan=True,
                          offset_preweight=True)
    gnp = [x.astype(np.float64) for x in geom]
    step = abs(float(angles[-1]) - float(angles[0])) / (A - 1)
    filt = oracle.fdk_filter(proj * w64[:, :, None], px, gnp[2], gnp[1], 0.8,
                             frame=(d64, u64, v64))
    truth = np.maximum(oracle.backproject(filt, gnp, px, shape, 1.0, off) * step, 0.0)
    assert rel_l2(vol.cpu(), truth) < 1e-5
