"""The forward projector's TMA arm (volume bricks staged in shared memory by
cp.async.bulk.tensor, fp_forward_tma_kernel) against its L1 arm
(fp_forward_kernel): bitwise the same projections -- both march the same
FP32 samples and sum them in the same order -- on small random geometries
(power-of-two and dividing voxel sizes, ROI offsets, thin volumes, rays
missing the volume, partial tiles), a detector so wide that bundles outgrow
the staged box (global fallback), and the configuration-2 geometry, for both
slab widths.  The arm is chosen through the library's arm rules
(dgc_fp_add_arm_rule), the way the autotuner registers its choice."""

import math

import numpy as np
import pytest
import torch

from test_gpu_forward import cuda32, random_case, run_project

pytestmark = pytest.mark.gpu


@pytest.fixture
def arm():
    from dgc_b200 import _native

    lib = _native.lib()

    def use(a, slab=0, unroll=1, view_block=0):
        _native.check(lib.dgc_fp_clear_arm_rules())
        if a is not None:
            _native.check(lib.dgc_fp_add_arm_rule(1 << 62, a, slab, unroll, view_block))

    use(None)
    yield use
    use(None)


CASES = {
    "pow2": dict(seed=11, vs=1.0, px=1.0, step=0.5, off=(0.0, 0.0, 0.0)),
    "div_offsets": dict(seed=12),
    "thin": dict(seed=13, shape=(3, 40, 5), vs=1.0, step=0.25),
    "wide_detector": dict(seed=14, U=200, V=90, px=0.7, vs=0.5, step=0.3),
    "odd_tiles": dict(seed=15, U=37, V=45, A=5),
}


@pytest.mark.parametrize("variant", [(1, 2, 1, 0), (1, 4, 1, 0), (0, 0, 2, 0), (0, 0, 1, 3),
                                     (2, 0, 1, 0), (2, 0, 1, 64)])
@pytest.mark.parametrize("name", sorted(CASES))
def test_tma_arm_is_bitwise_the_l1_arm(name, variant, arm):
    """TMA bricks (slab 2 or 4), the L1 arm's march unrolled twice, CTAs in
    view blocks, and the z-pair layout, each against the L1 arm unrolled once
    in the default order."""
    case = random_case(**CASES[name])
    arm(0)
    ref, _, _ = run_project(case)
    arm(*variant)
    got, _, _ = run_project(case)
    torch.cuda.synchronize()
    assert torch.isfinite(got).all()
    assert torch.equal(got, ref), float((got - ref).abs().max())


@pytest.mark.parametrize("variant", [(1, 2, 1, 0), (1, 4, 1, 0), (2, 0, 1, 0), (0, 0, 1, 16)])
def test_tma_arm_config2_views(variant, arm):
    """A 256^3 phantom, 24 views of config 2's scan (384^2, sid 1000, sod 600)."""
    from cbct_backprojector import project
    from dgc_b200.phantoms import circular_geometry, ellipsoid_phantom

    vol = ellipsoid_phantom((256, 256, 256), seed=3, device="cuda")
    geom = circular_geometry(24, 384, 384, 1000.0, 600.0, 1.0, device="cuda")
    geom[0] = geom[0] + 0.013  # off the axis-aligned angles
    arm(0)
    ref = project(vol, *geom, 1.0, 384, 384, step_size=0.5, voxel_size=1.0)
    arm(*variant)
    got = project(vol, *geom, 1.0, 384, 384, step_size=0.5, voxel_size=1.0)
    torch.cuda.synchronize()
    assert torch.equal(got, ref), float((got - ref).abs().max())


def test_arm_rules(arm):
    import ctypes

    from dgc_b200 import _native

    lib = _native.lib()
    out = [ctypes.c_int() for _ in range(4)]

    def query(D, H, W):
        _native.check(lib.dgc_fp_arm(D, H, W, *[ctypes.byref(x) for x in out]))
        return tuple(x.value for x in out)

    arm(None)
    assert query(64, 64, 64) == (0, 0, 1, 0)
    _native.check(lib.dgc_fp_add_arm_rule(100 ** 3, 1, 4, 1, 0))
    _native.check(lib.dgc_fp_add_arm_rule(600 ** 3, 0, 0, 2, 64))
    assert query(64, 64, 64) == (1, 4, 1, 0)
    assert query(512, 512, 512) == (0, 0, 2, 64)
    assert query(700, 700, 700) == (0, 0, 1, 16)  # built-in: view blocks above 2^26 voxels
    for bad in ((0, 0, 0, 1, 0), (10, 3, 0, 1, 0), (10, 1, 3, 1, 0), (10, 0, 0, 3, 0),
                (10, 1, 2, 2, 0), (10, 2, 0, 2, 0), (10, 0, 0, 1, -1)):
        with pytest.raises(RuntimeError):
            _native.check(lib.dgc_fp_add_arm_rule(*bad))
