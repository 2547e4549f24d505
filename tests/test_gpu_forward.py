"""Forward projector on the GPU: parity with the FP64 oracle, the reference's
own CUDA kernels and its CPU oracle (golden fixtures), gradients, edge cases.

Tolerances: the reference's check_forward_operator.py uses forward
rtol/atol 5e-5 and gradients rtol 1e-3 / atol 1e-4 against FP64; the
parity bar for this library is rel-L2 1e-5 for projections and 1e-4 for
gradients against the reference's CUDA path.
"""

import math

import numpy as np
import pytest
import torch

from conftest import GEOM_NAMES, golden_geometry, rel_l2

pytestmark = pytest.mark.gpu

FWD_RTOL = 1e-5   # rel-L2, projections
GRAD_RTOL = 1e-4  # rel-L2, gradients


def cuda32(x):
    return torch.as_tensor(np.asarray(x), dtype=torch.float32).cuda()


def noncontig(vol):
    """Same logical values, non-contiguous storage (as the reference's checks do)."""
    return vol.transpose(1, 2).contiguous().transpose(1, 2)


def random_case(seed, shape=(20, 28, 24), A=16, U=40, V=36, px=0.9, vs=0.8, step=0.37,
                off=(0.31, -0.22, 0.17)):
    rng = np.random.default_rng(seed)
    vol = rng.random(shape).astype(np.float32)
    angles = np.sort(rng.uniform(0, 2 * math.pi, A)).astype(np.float32)
    sid = (150 + rng.normal(0, 2, A)).astype(np.float32)
    sod = (95 + rng.normal(0, 1, A)).astype(np.float32)
    u0 = ((U - 1) / 2 + rng.normal(0, 1.5, A)).astype(np.float32)
    v0 = ((V - 1) / 2 + rng.normal(0, 1.5, A)).astype(np.float32)
    sx, sy, sz = (rng.normal(0, 0.6, A).astype(np.float32) for _ in range(3))
    geom = [angles, sid, sod, u0, v0, sx, sy, sz]
    return dict(vol=vol, geom=geom, px=px, U=U, V=V, step=step, vs=vs, off=off)


def run_project(case, vol=None, geom=None, requires_grad=False):
    from cbct_backprojector import project

    vol = cuda32(case["vol"]) if vol is None else vol
    geom = [cuda32(g) for g in case["geom"]] if geom is None else geom
    if requires_grad:
        vol.requires_grad_()
        for g in geom:
            g.requires_grad_()
    out = project(vol, *geom, case["px"], case["U"], case["V"], step_size=case["step"],
                  voxel_size=case["vs"], off_x=case["off"][0], off_y=case["off"][1],
                  off_z=case["off"][2])
    return out, vol, geom


# --------------------------------------------------------------- golden cases


def test_reference_check_case(golden):
    """examples/check_forward_operator.py case against its FP64 CPU oracle."""
    from cbct_backprojector import project

    d = golden("fp_check_case.npz")
    U, V = (int(x) for x in d["detector"])
    off = tuple(float(x) for x in d["volume_offset"])
    vol = noncontig(cuda32(d["in_data"])).requires_grad_()
    assert not vol.is_contiguous()
    geom = [cuda32(g).requires_grad_() for g in golden_geometry(d)]
    out = project(vol, *geom, float(d["pixel_size"]), U, V, step_size=float(d["step_size"]),
                  voxel_size=float(d["voxel_size"]), off_x=off[0], off_y=off[1], off_z=off[2])
    upstream = noncontig(cuda32(d["upstream"]))
    assert not upstream.is_contiguous()
    grads = torch.autograd.grad(out, [vol, *geom], grad_outputs=upstream)
    torch.testing.assert_close(out.double().cpu(), torch.from_numpy(d["output"]), rtol=5e-5,
                               atol=5e-5)
    for name, g in zip(("data",) + GEOM_NAMES, grads):
        assert torch.isfinite(g).all(), name
        torch.testing.assert_close(g.double().cpu(), torch.from_numpy(d["grad_" + name]),
                                   rtol=1e-3, atol=1e-4, msg=name)


def config1_case(d):
    U, V = (int(x) for x in d["detector"])
    return dict(vol=d["in_data"], geom=golden_geometry(d, np.float32), px=1.0, U=U, V=V,
                step=0.5, vs=1.0, off=(0.0, 0.0, 0.0))


def unambiguous_rays(oracle, case, shape):
    """1.0 for rays whose samples all sit > 1e-4 voxel from a cell boundary."""
    tr = oracle.ray_traces(shape, case["geom"], case["px"], case["U"], case["V"], case["step"],
                           case["vs"], case["off"], mode=1)
    return torch.tensor((tr != 0).astype(np.float32), device="cuda")


def test_config1_against_reference_cpu_oracle(golden, oracle):
    """Config 1 (16x20x24, 24 views, 48x40): values and loss=mean(p^2) gradients.

    The nominal config-1 geometry is grid-aligned: at 0/90/180/270 degrees about
    5 % of the rays have samples exactly on cell boundaries, where the
    piecewise-linear interpolant has kinks and FP32 and FP64 legitimately take
    different one-sided derivatives.  Geometry gradients are therefore checked
    strictly on the rays away from boundaries (the reference's own finite-
    difference check guards its ray the same way) and loosely in full.
    """
    d = golden("fp_config1.npz")
    case = config1_case(d)
    out, vol, geom = run_project(case, requires_grad=True)
    assert rel_l2(out.detach().cpu(), d["output"]) < FWD_RTOL
    p = out.detach().double()
    grads = torch.autograd.grad(out, [vol, *geom], grad_outputs=(2 * p / p.numel()).float(),
                                retain_graph=True)
    assert rel_l2(grads[0].cpu(), d["grad_data"]) < GRAD_RTOL
    for name, g in zip(GEOM_NAMES, grads[1:]):
        assert rel_l2(g.cpu(), d["grad_" + name]) < 5e-2, name
    mask = unambiguous_rays(oracle, case, d["in_data"].shape)
    up = (2 * p * mask / p.numel()).float()
    ours = torch.autograd.grad(out, geom, grad_outputs=up)
    _, gg = oracle.project_backward(up.cpu().numpy(), case["vol"], case["geom"], 1.0, 0.5, 1.0,
                                    mode=1, compute_grad_volume=False)
    for k, name in enumerate(GEOM_NAMES):
        assert rel_l2(ours[k].cpu(), gg[k]) < GRAD_RTOL, name


def test_config1_perturbed_geometry(golden, oracle):
    """Config 1 sizes with config-3 style per-view perturbations: strict FP64 check."""
    d = golden("fp_config1.npz")
    case = config1_case(d)
    rng = np.random.default_rng(31)
    A = len(case["geom"][0])
    g = [x.astype(np.float64) for x in case["geom"]]
    g[0] = g[0] + np.deg2rad(rng.normal(0, 0.3, A))
    g[1] = g[1] * (1 + rng.normal(0, 0.005, A))
    g[2] = g[2] * (1 + rng.normal(0, 0.005, A))
    g[3] = g[3] + rng.normal(0, 2, A)
    g[4] = g[4] + rng.normal(0, 2, A)
    for k in (5, 6, 7):
        g[k] = g[k] + rng.normal(0, 1.0, A)
    case["geom"] = [x.astype(np.float32) for x in g]
    out, vol, geom = run_project(case, requires_grad=True)
    truth = oracle.project(case["vol"], case["geom"], 1.0, case["U"], case["V"], 0.5, 1.0, mode=1)
    assert rel_l2(out.detach().cpu(), truth) < FWD_RTOL
    p = out.detach().double()
    mask = unambiguous_rays(oracle, case, d["in_data"].shape)
    up = (2 * p * mask / p.numel()).float()
    ours = torch.autograd.grad(out, [vol, *geom], grad_outputs=up)
    gv, gg = oracle.project_backward(up.cpu().numpy(), case["vol"], case["geom"], 1.0, 0.5, 1.0,
                                     mode=1)
    assert rel_l2(ours[0].cpu(), gv) < GRAD_RTOL
    for k, name in enumerate(GEOM_NAMES):
        assert rel_l2(ours[1 + k].cpu(), gg[k]) < GRAD_RTOL, name


# ------------------------------------------------------- reference CUDA parity


def _ref_forward(ref_fp, case):
    geom = [cuda32(g) for g in case["geom"]]
    return ref_fp.forward(cuda32(case["vol"]), *geom, case["px"], case["U"], case["V"],
                          case["step"], case["vs"], *case["off"])


@pytest.mark.parametrize("which", ["config1", "random_nonpow2", "random_pow2"])
def test_forward_matches_reference_cuda(which, golden, ref_native, oracle):
    ref_fp, _ = ref_native
    if which == "config1":
        case = config1_case(golden("fp_config1.npz"))
    elif which == "random_nonpow2":
        case = random_case(3)
    else:
        case = random_case(4, vs=0.5, px=1.0, step=0.25, off=(0.0, 0.0, 0.0))
    ours, _, _ = run_project(case)
    ref = _ref_forward(ref_fp, case)
    torch.cuda.synchronize()
    assert rel_l2(ours.cpu(), ref.cpu()) < FWD_RTOL
    # error against FP64 truth on the kernel's sample set
    truth = oracle.project(case["vol"], case["geom"], case["px"], case["U"], case["V"],
                           case["step"], case["vs"], case["off"], mode=1)
    assert rel_l2(ours.cpu(), truth) < FWD_RTOL


@pytest.mark.parametrize("which", ["config1", "random_nonpow2"])
def test_backward_matches_reference_cuda(which, golden, ref_native, oracle):
    """The volume gradient (run-merged level records folded afterwards) and
    the eight geometry gradients against the reference's CUDA and the FP64
    oracle."""
    ref_fp, _ = ref_native
    case = config1_case(golden("fp_config1.npz")) if which == "config1" else random_case(5)
    out, vol, geom = run_project(case, requires_grad=True)
    gp = (2.0 * out.detach() / out.numel()).contiguous()
    ours = torch.autograd.grad(out, [vol, *geom], grad_outputs=gp)
    ref = ref_fp.backward(gp, vol.detach(), *[g.detach() for g in geom], case["px"],
                          case["step"], case["vs"], True, *case["off"])
    torch.cuda.synchronize()
    for name, a, b in zip(("data",) + GEOM_NAMES, ours, ref):
        assert rel_l2(a.cpu(), b.cpu()) < GRAD_RTOL, name
    # FP64 truth on the rays whose samples stay away from cell boundaries
    mask = unambiguous_rays(oracle, case, case["vol"].shape)
    gpm = (gp * mask).contiguous()
    out2, vol2, geom2 = run_project(case, requires_grad=True)
    ours_m = torch.autograd.grad(out2, [vol2, *geom2], grad_outputs=gpm)
    gv, gg = oracle.project_backward(gpm.cpu().numpy(), case["vol"], case["geom"], case["px"],
                                     case["step"], case["vs"], case["off"], mode=1)
    assert rel_l2(ours_m[0].cpu(), gv) < GRAD_RTOL
    for k, name in enumerate(GEOM_NAMES):
        assert rel_l2(ours_m[1 + k].cpu(), gg[k]) < GRAD_RTOL, name


@pytest.mark.parametrize("shape", [(1, 1, 1), (1, 5, 4), (3, 1, 2), (2, 3, 1)])
def test_thin_volume_gradients(shape, oracle):
    """Volumes one or a few voxels thick: every padded corner folds onto an
    edge voxel, the records' z range is at its smallest.  Volume gradient
    against the FP64 oracle."""
    case = random_case(31, shape=shape, A=6, U=12, V=10, vs=1.0, step=0.25, off=(0.1, -0.2, 0.05))
    out, vol, geom = run_project(case, requires_grad=True)
    up = torch.linspace(0.2, 1.1, out.numel(), device="cuda").view_as(out)
    (gv,) = torch.autograd.grad(out, [vol], grad_outputs=up)
    truth, _ = oracle.project_backward(up.cpu().numpy(), case["vol"], case["geom"], case["px"],
                                       case["step"], case["vs"], case["off"], mode=1)
    assert float(np.abs(truth).sum()) > 0.0
    assert rel_l2(gv.cpu(), truth) < GRAD_RTOL


# ----------------------------------------------------------- finite differences


def test_config1_finite_differences(golden, oracle):
    """Central differences of L = mean(p^2) for voxels (eps=1e-3) and src_x.

    For a geometry parameter the loss runs over the rays whose trace (entry
    face, sample count, interpolation cells; oracle.ray_traces) is the same at
    the base point and at +-eps, i.e. the difference stays inside one smooth
    piece -- the guard of the reference's check_forward_operator.py:178-193.
    The src_x step is 1e-2: sample offsets t_k come from the FP32 recurrence
    and are quantised to ~1e-5, which at eps=1e-3 is a few percent of the
    displacement a source shift produces (the FP64 oracle shows the same).
    """
    from dgc_b200 import _ops

    d = golden("fp_config1.npz")
    case = config1_case(d)
    shape = d["in_data"].shape
    out, vol, geom = run_project(case, requires_grad=True)
    p = out.detach().double()
    gvol = torch.autograd.grad(out, vol, grad_outputs=(2 * p / p.numel()).float(),
                               retain_graph=True)[0]
    eps = 1e-3
    base = vol.detach()
    for i in torch.topk(gvol.abs().flatten(), 3).indices.tolist():
        e = torch.zeros_like(base).flatten()
        e[i] = eps
        e = e.view_as(base)
        lp = run_project(case, vol=base + e)[0].double().square().mean()
        lm = run_project(case, vol=base - e)[0].double().square().mean()
        fd = ((lp - lm) / (2 * eps)).item()
        assert math.isclose(gvol.flatten()[i].item(), fd, rel_tol=1e-2, abs_tol=1e-6)

    k_sx = GEOM_NAMES.index("src_x")
    eps = 1e-2
    t0 = oracle.ray_traces(shape, case["geom"], 1.0, case["U"], case["V"], 0.5, 1.0, mode=1)
    for a in (1, 5, 13, 22):
        gplus = [g.detach().clone() for g in geom]
        gminus = [g.detach().clone() for g in geom]
        gplus[k_sx][a] += eps
        gminus[k_sx][a] -= eps
        tp = oracle.ray_traces(shape, [g.cpu().numpy() for g in gplus], 1.0, case["U"], case["V"],
                               0.5, 1.0, mode=1)
        tm = oracle.ray_traces(shape, [g.cpu().numpy() for g in gminus], 1.0, case["U"],
                               case["V"], 0.5, 1.0, mode=1)
        c0 = _ops.project_sample_counts(shape, [g.detach() for g in geom], 1.0, case["U"],
                                        case["V"], 0.5, 1.0).cpu().numpy()
        cp = _ops.project_sample_counts(shape, gplus, 1.0, case["U"], case["V"], 0.5, 1.0)
        cm = _ops.project_sample_counts(shape, gminus, 1.0, case["U"], case["V"], 0.5, 1.0)
        keep = ((t0 != 0) & (t0 == tp) & (t0 == tm) & (cp.cpu().numpy() == c0) &
                (cm.cpu().numpy() == c0))
        assert keep[a].mean() > 0.5
        mask = torch.tensor(keep.astype(np.float64), device="cuda")
        upstream = (2 * p * mask / p.numel()).float()
        g = torch.autograd.grad(out, geom[k_sx], grad_outputs=upstream, retain_graph=True)[0]
        fp_ = (run_project(case, geom=gplus)[0].double().square() * mask).sum() / p.numel()
        fm_ = (run_project(case, geom=gminus)[0].double().square() * mask).sum() / p.numel()
        denom = (gplus[k_sx][a] - gminus[k_sx][a]).item()
        fd = ((fp_ - fm_) / denom).item()
        assert math.isclose(g[a].item(), fd, rel_tol=1e-2, abs_tol=1e-5), (a, g[a].item(), fd)


# ------------------------------------------------------------- properties, edges


def test_linearity_and_determinism():
    case = random_case(11)
    a = cuda32(case["vol"])
    b = a.flip(-1).contiguous()
    pa, _, _ = run_project(case, vol=a)
    pb, _, _ = run_project(case, vol=b)
    pc, _, _ = run_project(case, vol=1.3 * a - 0.4 * b)
    torch.testing.assert_close(pc, 1.3 * pa - 0.4 * pb, rtol=5e-5, atol=5e-5)
    # geometry gradients are reduced in a fixed order: bitwise reproducible
    outs = []
    for _ in range(2):
        out, vol, geom = run_project(case, requires_grad=True)
        outs.append(torch.autograd.grad(out.square().sum(), geom))
    for g1, g2 in zip(*outs):
        assert torch.equal(g1, g2)


def test_edge_cases(oracle):
    from cbct_backprojector import project

    # single ray, single view, 1x1x1 volume
    case = dict(vol=np.full((1, 1, 1), 2.0, np.float32),
                geom=[np.zeros(1, np.float32), np.full(1, 50.0, np.float32),
                      np.full(1, 30.0, np.float32), np.zeros(1, np.float32),
                      np.zeros(1, np.float32), np.zeros(1, np.float32), np.zeros(1, np.float32),
                      np.zeros(1, np.float32)],
                px=1.0, U=1, V=1, step=0.1, vs=1.0, off=(0.0, 0.0, 0.0))
    out, _, _ = run_project(case)
    truth = oracle.project(case["vol"], case["geom"], 1.0, 1, 1, 0.1, 1.0, mode=1)
    assert rel_l2(out.cpu(), truth) < FWD_RTOL and out.item() > 0
    # detector shifted off the volume: every ray misses, all zero
    case2 = random_case(21)
    case2["geom"][3] = case2["geom"][3] + 5000.0
    out2, vol, geom = run_project(case2, requires_grad=True)
    assert torch.count_nonzero(out2) == 0
    grads = torch.autograd.grad(out2.sum(), [vol, *geom])
    assert all(torch.count_nonzero(g) == 0 for g in grads)
    # zero upstream gradient on a subset of rays -> those rays contribute nothing
    case3 = random_case(22)
    out3, vol3, geom3 = run_project(case3, requires_grad=True)
    up = torch.zeros_like(out3)
    up[0] = 1.0
    g3 = torch.autograd.grad(out3, [vol3, *geom3], grad_outputs=up)
    assert torch.count_nonzero(g3[1][1:]) == 0
    assert torch.isfinite(g3[0]).all()
    # only the views that exist, shape check, and direct apply without ROI args
    from cbct_backprojector import DifferentiableSourceOnlyForwardProjector as F

    vol4 = cuda32(case3["vol"]).requires_grad_()
    geom4 = [cuda32(g) for g in case3["geom"]]
    y = F.apply(vol4, *geom4, case3["px"], case3["U"], case3["V"], case3["step"], case3["vs"])
    assert y.shape == (16, case3["U"], case3["V"])
    (gv,) = torch.autograd.grad(y.sum(), vol4)
    assert torch.isfinite(gv).all()
    # non-contiguous geometry tensors
    geom5 = [torch.stack([g, g], 1)[:, 0] for g in geom4]
    assert not geom5[0].is_contiguous()
    y5 = project(cuda32(case3["vol"]), *geom5, case3["px"], case3["U"], case3["V"],
                 step_size=case3["step"], voxel_size=case3["vs"])
    y4 = project(cuda32(case3["vol"]), *geom4, case3["px"], case3["U"], case3["V"],
                 step_size=case3["step"], voxel_size=case3["vs"])
    assert torch.equal(y4, y5)
