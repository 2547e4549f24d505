"""Backprojector on the GPU: parity with the reference's CPU oracle (golden
fixtures), the reference's own CUDA kernels and the FP64 oracle; gradients;
edge cases.

Tolerances: the reference's check_operator.py uses forward rtol/atol 2e-5 and
gradients rtol 3e-4 / atol 3e-5 against FP64; the parity bar of this library
is rel-L2 1e-5 (values) and 1e-4 (gradients) against the reference's CUDA.
"""

import math

import numpy as np
import pytest
import torch

from conftest import GEOM_NAMES, golden_geometry, rel_l2

pytestmark = pytest.mark.gpu

FWD_RTOL = 1e-5
GRAD_RTOL = 1e-4


def cuda32(x):
    return torch.as_tensor(np.asarray(x), dtype=torch.float32).cuda()


def random_case(seed, A=24, U=48, V=40, shape=(18, 22, 26), px=0.9, vs=0.8,
                off=(0.27, -0.31, 0.23)):
    rng = np.random.default_rng(seed)
    proj = rng.random((A, U, V)).astype(np.float32) * 2 - 0.5
    angles = (np.arange(A) * 2 * math.pi / A + rng.normal(0, 0.01, A)).astype(np.float32)
    sid = (180 + rng.normal(0, 2, A)).astype(np.float32)
    sod = (120 + rng.normal(0, 1, A)).astype(np.float32)
    u0 = ((U - 1) / 2 + rng.normal(0, 1.5, A)).astype(np.float32)
    v0 = ((V - 1) / 2 + rng.normal(0, 1.5, A)).astype(np.float32)
    sx, sy, sz = (rng.normal(0, 0.6, A).astype(np.float32) for _ in range(3))
    return dict(proj=proj, geom=[angles, sid, sod, u0, v0, sx, sy, sz], px=px,
                shape=shape, vs=vs, off=off)


def run_bp(case, requires_grad=False):
    from cbct_backprojector import backproject

    proj = cuda32(case["proj"])
    geom = [cuda32(g) for g in case["geom"]]
    if requires_grad:
        proj.requires_grad_()
        for g in geom:
            g.requires_grad_()
    vol = backproject(proj, *geom, case["px"], case["shape"], case["vs"],
                      volume_offset=case["off"])
    return vol, proj, geom


def test_reference_check_case(golden):
    """examples/check_operator.py case (non-contiguous inputs) against its FP64 oracle."""
    from cbct_backprojector import backproject

    d = golden("bp_check_case.npz")
    proj = cuda32(d["in_data"]).transpose(1, 2).contiguous().transpose(1, 2).requires_grad_()
    assert not proj.is_contiguous()
    geom = [cuda32(g).requires_grad_() for g in golden_geometry(d)]
    upstream = cuda32(d["upstream"]).transpose(1, 2).contiguous().transpose(1, 2)
    shape = tuple(int(s) for s in d["volume_shape"])
    vol = backproject(proj, *geom, float(d["pixel_size"]), shape, float(d["voxel_size"]),
                      volume_offset=tuple(float(x) for x in d["volume_offset"]))
    grads = torch.autograd.grad(vol, [proj, *geom], grad_outputs=upstream)
    torch.testing.assert_close(vol.double().cpu(), torch.from_numpy(d["output"]), rtol=2e-5,
                               atol=2e-5)
    for name, g in zip(("data",) + GEOM_NAMES, grads):
        torch.testing.assert_close(g.double().cpu(), torch.from_numpy(d["grad_" + name]),
                                   rtol=3e-4, atol=3e-5, msg=name)


def test_config1_against_reference_cpu_oracle(golden, ref_native):
    """Config-1 backprojection (24 views of 48x40 into 16x20x24).

    The nominal geometry is grid-aligned (voxel centres project exactly onto
    detector-pixel boundaries at several views), where the bilinear weights'
    derivatives jump; FP32 and FP64 pick different sides there, so geometry
    gradients are compared with the FP64 golden loosely and with the
    reference's CUDA (same FP32 rounding of the mapping) strictly.
    """
    _, ref_bp = ref_native
    d = golden("bp_config1.npz")
    case = dict(proj=d["in_data"], geom=golden_geometry(d, np.float32), px=1.0,
                shape=tuple(int(s) for s in d["volume_shape"]), vs=1.0, off=(0.0, 0.0, 0.0))
    vol, proj, geom = run_bp(case, requires_grad=True)
    assert rel_l2(vol.detach().cpu(), d["output"]) < FWD_RTOL
    up = cuda32(d["upstream"])
    grads = torch.autograd.grad(vol, [proj, *geom], grad_outputs=up)
    assert rel_l2(grads[0].cpu(), d["grad_data"]) < GRAD_RTOL
    for name, g in zip(GEOM_NAMES, grads[1:]):
        assert rel_l2(g.cpu(), d["grad_" + name]) < 5e-2, name
    ref = ref_bp.forward(proj.detach(), *[g.detach() for g in geom], 1.0, *case["shape"], 1.0)
    theirs = ref_bp.backward(up, proj.detach(), *[g.detach() for g in geom], 1.0, 1.0)
    torch.cuda.synchronize()
    assert rel_l2(vol.detach().cpu(), ref.cpu()) < FWD_RTOL
    for k, name in enumerate(("data",) + GEOM_NAMES):
        assert rel_l2(grads[k].cpu(), theirs[k].cpu()) < GRAD_RTOL, name


@pytest.mark.parametrize("seed,px,vs,shape", [(1, 0.9, 0.8, (18, 22, 26)),
                                             (2, 1.0, 1.0, (40, 33, 29)),
                                             (3, 0.5, 0.75, (70, 24, 20))])
def test_matches_reference_cuda(seed, px, vs, shape, ref_native, oracle):
    _, ref_bp = ref_native
    case = random_case(seed, px=px, vs=vs, shape=shape)
    vol, proj, geom = run_bp(case, requires_grad=True)
    ref = ref_bp.forward(proj.detach(), *[g.detach() for g in geom], px, *shape, vs, *case["off"])
    torch.cuda.synchronize()
    assert rel_l2(vol.detach().cpu(), ref.cpu()) < FWD_RTOL
    truth = oracle.backproject(case["proj"], case["geom"], px, shape, vs, case["off"])
    assert rel_l2(vol.detach().cpu(), truth) < FWD_RTOL
    up = torch.linspace(-0.7, 1.3, vol.numel(), device="cuda").view_as(vol)
    ours = torch.autograd.grad(vol, [proj, *geom], grad_outputs=up)
    theirs = ref_bp.backward(up, proj.detach(), *[g.detach() for g in geom], px, vs, *case["off"])
    gp, gg = oracle.backproject_backward(up.cpu().numpy(), case["proj"], case["geom"], px, vs,
                                         case["off"])
    torch.cuda.synchronize()
    for k, name in enumerate(("data",) + GEOM_NAMES):
        assert rel_l2(ours[k].cpu(), theirs[k].cpu()) < GRAD_RTOL, name
        truth_k = gp if k == 0 else gg[k - 1]
        assert rel_l2(ours[k].cpu(), truth_k) < GRAD_RTOL, name


def test_determinism_and_edges():
    case = random_case(7)
    outs = []
    for _ in range(2):
        vol, proj, geom = run_bp(case, requires_grad=True)
        outs.append(torch.autograd.grad(vol.square().sum(), geom))
    for a, b in zip(*outs):
        assert torch.equal(a, b)
    # a volume entirely outside the detector's view: zero output and gradients
    far = dict(case, off=(0.0, 0.0, 5000.0))
    vol, proj, geom = run_bp(far, requires_grad=True)
    assert torch.count_nonzero(vol) == 0
    grads = torch.autograd.grad(vol.sum(), [proj, *geom])
    assert all(torch.count_nonzero(g) == 0 for g in grads)
    # minimum detector (U = V = 2) and a single view and voxel
    tiny = dict(proj=np.ones((1, 2, 2), np.float32),
                geom=[np.zeros(1, np.float32), np.full(1, 20.0, np.float32),
                      np.full(1, 10.0, np.float32), np.full(1, 0.5, np.float32),
                      np.full(1, 0.5, np.float32)] + [np.zeros(1, np.float32)] * 3,
                px=1.0, shape=(1, 1, 1), vs=0.1, off=(0.0, 0.0, 0.0))
    v, _, _ = run_bp(tiny)
    # voxel at (-0.05, -0.05, -0.05): weight ((sod)/(sod+0.05))^2, bilinear of ones = 1
    q = 10.0 + 0.05
    assert math.isclose(v.item(), (10.0 / q) ** 2, rel_tol=1e-5)


def test_geometry_only_backward_skips_the_projection_gradient():
    """With projections that need no gradient the scatter is skipped
    (grad_projections NULL in the C ABI); the geometry gradients are bitwise
    those of the full backward."""
    from dgc_b200 import _ops

    case = random_case(5)
    vol, proj, geom = run_bp(case, requires_grad=True)
    up = torch.linspace(-0.7, 1.3, vol.numel(), device="cuda").view_as(vol)
    full = torch.autograd.grad(vol, [proj, *geom], grad_outputs=up)
    from cbct_backprojector import backproject

    geom2 = [cuda32(g).requires_grad_() for g in case["geom"]]
    vol2 = backproject(cuda32(case["proj"]), *geom2, case["px"], case["shape"], case["vs"],
                       volume_offset=case["off"])
    part = torch.autograd.grad(vol2, geom2, grad_outputs=up)
    for a, b in zip(full[1:], part):
        assert torch.equal(a, b)
    grads = _ops.bp_backward(up, proj.detach(), *[g.detach() for g in geom], case["px"], case["vs"],
                             *case["off"], compute_grad_proj=False)
    assert grads[0] is None
    for a, b in zip(full[1:], grads[1:]):
        assert torch.equal(a, b)


@pytest.fixture
def tile_rule():
    """Sets one library tile rule for every backprojection (dgc_bp_add_tile_rule)
    and clears the rules afterwards."""
    from dgc_b200 import _native

    lib = _native.lib()

    def set_rule(kz=0, cta=(0, 0)):
        _native.check(lib.dgc_bp_clear_tile_rules())
        _native.check(lib.dgc_bp_add_tile_rule(1 << 30, 1 << 30, kz, kz, cta[0], cta[1]))

    lib.dgc_bp_clear_tile_rules()
    yield set_rule
    lib.dgc_bp_clear_tile_rules()


@pytest.mark.parametrize("px", [1.0, 0.9])
@pytest.mark.parametrize("kz", [1, 2, 4, 8])
def test_every_z_blocking_matches_the_oracle(kz, px, oracle, tile_rule):
    """32*KZ voxels of a column per warp (the defaults pick 2 for the forward,
    4 for the backward; the autotuner may pick any): every choice, with D not
    a multiple of the warp's span and with the dividing (non power-of-two)
    pixel size, against the FP64 oracle."""
    tile_rule(kz=kz)
    case = random_case(4, px=px, vs=1.0, shape=(70, 21, 19))
    vol, proj, geom = run_bp(case, requires_grad=True)
    truth = oracle.backproject(case["proj"], case["geom"], px, case["shape"], 1.0, case["off"])
    assert rel_l2(vol.detach().cpu(), truth) < FWD_RTOL
    up = torch.linspace(-0.7, 1.3, vol.numel(), device="cuda").view_as(vol)
    ours = torch.autograd.grad(vol, [proj, *geom], grad_outputs=up)
    gp, gg = oracle.backproject_backward(up.cpu().numpy(), case["proj"], case["geom"], px, 1.0,
                                         case["off"])
    assert rel_l2(ours[0].cpu(), gp) < GRAD_RTOL
    for k, name in enumerate(GEOM_NAMES):
        assert rel_l2(ours[1 + k].cpu(), gg[k]) < GRAD_RTOL, name


@pytest.mark.parametrize("cta", [(4, 2), (2, 4), (4, 4), (16, 1), (3, 5)])
def test_column_patch_shapes_are_bitwise(cta, tile_rule):
    """The forward's CTA as a cx x cy patch of columns (a tile rule) gives the
    default's volume bit for bit (each voxel sums its views in one order),
    W and H not multiples of the patch included."""
    from cbct_backprojector import backproject

    case = random_case(6, px=1.0, vs=1.0, shape=(45, 23, 19))
    proj = cuda32(case["proj"])
    geom = [cuda32(g) for g in case["geom"]]
    a = backproject(proj, *geom, 1.0, case["shape"], 1.0, volume_offset=case["off"])
    tile_rule(cta=cta)
    b = backproject(proj, *geom, 1.0, case["shape"], 1.0, volume_offset=case["off"])
    torch.cuda.synchronize()
    assert torch.equal(a, b)


def test_autotuner_on_backprojector(tmp_path):
    """tune_backprojector on the GPU: every candidate timed, the choice
    registered as a library rule, the volume unchanged bit for bit."""
    from dgc_b200 import _native, backproject
    from dgc_b200.autotune import Autotuner, backprojector_tiles

    lib = _native.lib()
    lib.dgc_bp_clear_tile_rules()
    try:
        case = random_case(8, px=1.0, vs=1.0, shape=(70, 21, 19))
        proj = cuda32(case["proj"])
        geom = [cuda32(g) for g in case["geom"]]
        base = backproject(proj, *geom, 1.0, case["shape"], 1.0, volume_offset=case["off"])
        tuner = Autotuner(cache_path=tmp_path / "tiles.json")
        e = tuner.tune_backprojector(proj, geom, 1.0, case["shape"], 1.0, case["off"])
        assert len(e["forward_ms"]) == 8 and len(e["backward_ms"]) == 3
        assert backprojector_tiles(70, proj.shape[0]) == (e["kz_forward"], e["kz_backward"],
                                                          tuple(e["cta"]))
        tuned = backproject(proj, *geom, 1.0, case["shape"], 1.0, volume_offset=case["off"])
        torch.cuda.synchronize()
        assert torch.equal(base, tuned)
    finally:
        lib.dgc_bp_clear_tile_rules()


@pytest.mark.parametrize("shape", [(1, 1, 1), (1, 7, 5), (5, 1, 3), (33, 2, 2), (65, 3, 9)])
def test_thin_volumes(shape, oracle):
    """Volumes one or a few voxels thick along an axis (partial column
    patches, partial Z blocks): values and all nine gradients against the
    FP64 oracle."""
    case = random_case(9, px=1.0, vs=1.0, shape=shape)
    vol, proj, geom = run_bp(case, requires_grad=True)
    truth = oracle.backproject(case["proj"], case["geom"], 1.0, shape, 1.0, case["off"])
    assert rel_l2(vol.detach().cpu(), truth) < FWD_RTOL
    up = torch.linspace(0.3, 1.2, vol.numel(), device="cuda").view_as(vol)
    ours = torch.autograd.grad(vol, [proj, *geom], grad_outputs=up)
    gp, gg = oracle.backproject_backward(up.cpu().numpy(), case["proj"], case["geom"], 1.0, 1.0,
                                         case["off"])
    assert rel_l2(ours[0].cpu(), gp) < GRAD_RTOL
    for k, name in enumerate(GEOM_NAMES):
        assert rel_l2(ours[1 + k].cpu(), gg[k]) < GRAD_RTOL, name
