"""Host side of the batched projection without a GPU: the ctypes mirror of
``dgc_fp_instance`` / ``dgc_batch_plan`` matches the library (the workspace
query reads the fields it needs), argument checks name the failing instance
before any CUDA call, and the autotuner's buckets and JSON cache."""

import ctypes
import math
from types import SimpleNamespace

import pytest


def _instances(specs, grad_volume=True):
    from dgc_b200 import _native

    arr = (_native.FpInstance * len(specs))()
    for inst, (D, H, W, A, U, V, tb) in zip(arr, specs):
        inst.D, inst.H, inst.W, inst.A, inst.U, inst.V = D, H, W, A, U, V
        inst.pixel_size = inst.step_size = inst.voxel_size = 1.0
        for name in ("volume", "angles", "sid", "sod", "det_u0", "det_v0", "src_x", "src_y",
                     "src_z", "projections", "grad_projections", "grad_geometry"):
            setattr(inst, name, 256)
        inst.grad_volume = 256 if grad_volume else None
        inst.tile_backward = tb
    return arr


def _align(n):
    return (n + 255) // 256 * 256


def test_workspace_bytes_follow_the_layout():
    """Volume-gradient buffers: 16-byte level records over (D+2)(H+1)(W+1)
    cells."""
    from dgc_b200 import _native

    lib = _native.lib()
    specs = [(24, 20, 16, 12, 40, 36, 8), (9, 31, 27, 7, 33, 65, 4), (5, 7, 6, 33, 12, 9, 0)]
    for gv in (True, False):
        got = lib.dgc_batch_workspace_bytes(_instances(specs, gv), len(specs))
        per = 0
        for D, H, W, A, U, V, tb in specs:
            tu = tb or 8
            tiles = math.ceil(U / tu) * math.ceil(V / (256 // tu))
            per += _align(16 * (D + 2) * (H + 1) * (W + 1)) + _align(8 * 8 * A * tiles)
            if gv:
                per += _align(16 * (D + 2) * (H + 1) * (W + 1))
        n = len(specs)
        table = got - per - 5 * _align(8 * (n + 1)) - _align(16)
        # the n device-side instance records precede the buffers
        assert table % 256 == 0 and 64 * n <= table <= 512 * n
    assert lib.dgc_batch_workspace_bytes(None, 0) == 0
    bad = _instances([(0, 4, 4, 1, 4, 4, 0)])
    assert lib.dgc_batch_workspace_bytes(bad, 1) == 0


def test_prepare_rejects_bad_instances():
    from dgc_b200 import _native

    lib = _native.lib()
    plan = _native.BatchPlan()
    arr = _instances([(8, 8, 8, 4, 16, 16, 0), (8, 8, 8, 4, 0, 16, 0)])
    rc = lib.dgc_batch_prepare(arr, 2, None, 0, ctypes.byref(plan), None)
    assert rc == 1 and lib.dgc_last_error() == b"instance 1: U and V must be positive"
    arr = _instances([(8, 8, 8, 4, 16, 16, 0)])
    arr[0].tile_forward = 16
    rc = lib.dgc_batch_prepare(arr, 1, None, 0, ctypes.byref(plan), None)
    assert rc == 1 and b"tile_forward" in lib.dgc_last_error()
    arr[0].tile_forward = 2
    arr[0].tile_backward = 2
    rc = lib.dgc_batch_prepare(arr, 1, None, 0, ctypes.byref(plan), None)
    assert rc == 1 and b"tile_backward" in lib.dgc_last_error()
    arr[0].tile_backward = 4
    rc = lib.dgc_batch_prepare(arr, 1, None, 0, ctypes.byref(plan), None)
    assert rc == 3 and b"workspace" in lib.dgc_last_error()
    rc = lib.dgc_batch_prepare(arr, 0, None, 0, ctypes.byref(plan), None)
    assert rc == 1
    rc = lib.dgc_batch_project(ctypes.byref(_native.BatchPlan()), None)
    assert rc == 1 and b"prepared" in lib.dgc_last_error()


def _problem(shape, A, U, V, voxel=1.0):
    return SimpleNamespace(volume=SimpleNamespace(shape=shape),
                           geometry=[SimpleNamespace(numel=lambda A=A: A)] * 8, U=U, V=V,
                           voxel_size=voxel, tiles=(0, 0))


def test_buckets():
    from dgc_b200.autotune import bucket

    a = bucket(_problem((256, 256, 256), 360, 384, 384))
    assert a == "vol2^24-U384-V384-mul"
    assert bucket(_problem((250, 256, 256), 720, 380, 300)) == "vol2^24-U384-V384-mul"
    assert bucket(_problem((256, 256, 256), 360, 384, 384, voxel=0.75)).endswith("-div")
    assert bucket(_problem((128, 128, 128), 90, 512, 512)) == "vol2^21-U512-V512-mul"


def test_autotuner_picks_fastest_and_caches(tmp_path):
    from dgc_b200.autotune import Autotuner

    calls = []

    def fake(pr, direction, tile):
        calls.append((direction, tile))
        best = 4 if direction == "forward" else 8
        return 1.0 if tile == best else 2.0 + tile

    path = tmp_path / "t.json"
    tuner = Autotuner(cache_path=path, measure=fake)
    probs = [_problem((64, 64, 64), 90, 256, 256), _problem((64, 64, 64), 90, 256, 256),
             _problem((96, 96, 64), 180, 384, 256)]
    assert tuner.choose(probs) == [(4, 8)] * 3
    assert len(tuner.measured) == 2 and len(calls) == 2 * (3 + 2)
    again = Autotuner(cache_path=path, measure=lambda *a: pytest.fail("cache miss"))
    assert again.choose(probs) == [(4, 8)] * 3
    assert probs[2].tiles == (4, 8)


@pytest.fixture
def clean_bp_rules():
    from dgc_b200 import _native

    lib = _native.lib()
    lib.dgc_bp_clear_tile_rules()
    yield lib
    lib.dgc_bp_clear_tile_rules()


def test_backprojector_tile_rules(clean_bp_rules):
    """Built-in Z blocking, rules (first match, zero fields keep the built-in
    choice) and argument checks -- host only."""
    from dgc_b200 import _native
    from dgc_b200.autotune import backprojector_tiles

    lib = clean_bp_rules
    assert backprojector_tiles(256, 360) == (2, 4, (8, 1))
    assert backprojector_tiles(50, 90) == (2, 2, (8, 1))
    assert backprojector_tiles(20, 10) == (1, 1, (8, 1))
    assert lib.dgc_bp_add_tile_rule(64, 128, 1, 0, 0, 0) == 0
    assert lib.dgc_bp_add_tile_rule(256, 512, 8, 8, 4, 2) == 0
    assert backprojector_tiles(50, 90) == (1, 2, (8, 1))       # first rule; kz_backward built in
    assert backprojector_tiles(256, 360) == (8, 8, (4, 2))     # second rule
    assert backprojector_tiles(256, 600) == (2, 4, (8, 1))     # no rule covers A = 600
    for bad in ((0, 10, 2, 2, 0, 0), (64, 10, 3, 2, 0, 0), (64, 10, 2, 2, 5, 4),
                (64, 10, 2, 2, 4, 0)):
        with pytest.raises(RuntimeError):
            _native.check(lib.dgc_bp_add_tile_rule(*bad))
    for _ in range(14):
        assert lib.dgc_bp_add_tile_rule(1024, 1024, 2, 4, 0, 0) == 0
    with pytest.raises(RuntimeError, match="full"):
        _native.check(lib.dgc_bp_add_tile_rule(1024, 1024, 2, 4, 0, 0))


def test_autotuner_tunes_backprojector(clean_bp_rules, tmp_path):
    """Fastest forward (KZ, patch) and backward KZ per (depth, views) bucket,
    cached as JSON and registered as a library rule."""
    from dgc_b200.autotune import Autotuner, backprojector_tiles, bp_bucket

    assert bp_bucket((256, 256, 256), 360) == (256, 512)
    assert bp_bucket((100, 8, 8), 1) == (128, 1)
    calls = []

    def fake(proj, geom, px, shape, vs, off, direction, kz, cta):
        calls.append((direction, kz, tuple(cta)))
        if direction == "forward":
            return 1.0 + abs(kz - 4) + (0.5 if tuple(cta) == (8, 1) else 0.0)
        return 1.0 + abs(kz - 8)

    geom = [SimpleNamespace(numel=lambda: 360)]
    path = tmp_path / "tiles.json"
    tuner = Autotuner(cache_path=path, measure_bp=fake)
    e = tuner.tune_backprojector(None, geom, 1.0, (256, 256, 256), 1.0)
    assert (e["kz_forward"], e["kz_backward"], e["cta"]) == (4, 8, [4, 2])
    assert len(calls) == 4 * 2 + 3
    assert backprojector_tiles(256, 360) == (4, 8, (4, 2))
    clean_bp_rules.dgc_bp_clear_tile_rules()
    again = Autotuner(cache_path=path, measure_bp=lambda *a: pytest.fail("cache miss"))
    assert again.tune_backprojector(None, geom, 1.0, (200, 9, 9), 1.0)["kz_forward"] == 4
    assert backprojector_tiles(256, 360) == (4, 8, (4, 2))


def test_autotuner_tunes_forward_arm(tmp_path):
    """Fastest forward arm (L1 quads or TMA bricks, slab 2 or 4) per
    volume-size bucket, cached as JSON and registered as a library arm rule;
    a second tuner answers from the cache -- host only."""
    import ctypes

    from dgc_b200 import _native
    from dgc_b200.autotune import FORWARD_ARMS, Autotuner, arm_bucket

    lib = _native.lib()
    lib.dgc_fp_clear_arm_rules()
    try:
        assert arm_bucket((256, 256, 256)) == 1 << 24
        assert arm_bucket((100, 20, 20)) == 1 << 16
        calls = []

        def fake(problem, arm, slab, unroll, view_block):
            calls.append((arm, slab, unroll, view_block))
            return 2.0 if (arm, slab) == (1, 4) else 3.0 + 0.1 * arm + 0.01 * view_block

        pr = SimpleNamespace(volume=SimpleNamespace(shape=(512, 512, 512)))
        path = tmp_path / "tiles.json"
        e = Autotuner(cache_path=path, measure_arm=fake).tune_forward_arm(pr)
        assert (e["arm"], e["slab"], e["arm_name"]) == (1, 4, "tma-slab4")
        assert sorted(calls) == sorted(FORWARD_ARMS)
        out = [ctypes.c_int() for _ in range(4)]

        def query(D, H, W):
            _native.check(lib.dgc_fp_arm(D, H, W, *[ctypes.byref(x) for x in out]))
            return tuple(x.value for x in out)

        assert query(512, 512, 512) == (1, 4, 1, 0)
        # beyond every bucket: the built-in choice (L1 arm; view blocks of 16 above 2^26 voxels)
        assert query(600, 512, 512) == (0, 0, 1, 16)
        lib.dgc_fp_clear_arm_rules()
        again = Autotuner(cache_path=path, measure_arm=lambda *x: pytest.fail("cache miss"))
        assert again.tune_forward_arm(pr)["arm"] == 1
        assert query(512, 512, 512) == (1, 4, 1, 0)
    finally:
        lib.dgc_fp_clear_arm_rules()
