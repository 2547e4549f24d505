"""Tile autotuner of the forward projector and its backward.

The ray kernels run 256 rays per CTA as TU detector columns x 256/TU rows
(the 32 lanes of a warp along detector V).  Which TU is fastest depends on the
detector and volume shape: narrow tiles keep more rows of one column together
(better z-locality of the volume reads), wide tiles share more of a view's
volume slab across columns.  The tuner times every candidate on a
representative problem of each shape bucket, with CUDA events, and keeps the
choice in a JSON cache so that a bucket is measured once per machine.

Buckets: volume size class (log2 of the voxel count, rounded), detector U and
V rounded up to a multiple of 128, and whether the voxel size is a power of
two (division or multiplication variant).  The view count only scales the
number of tiles, so it is not part of the key, and a bucket is timed on its
first ``TUNE_VIEWS`` views.

The forward projector of a single problem also has two arms
(``tune_forward_arm``): quad loads through L1 (``fp_forward_kernel``, its march
loop unrolled once or twice), volume bricks staged in shared memory by TMA,
slabs of 2 or 4 cells along the ray bundle (``fp_forward_tma_kernel``), or the
volume as z pairs, half the quads' bytes (``fp_forward_pairs_kernel``); and the
order of the CTAs (every u tile of a view first, or views in blocks).  All
give bitwise the same projections; the fastest per volume-size bucket (voxel
count rounded up to a power of two) is registered in the library as an arm
rule (``dgc_fp_add_arm_rule``).

The backprojector is tuned the same way (``tune_backprojector``): the Z
blocking of its forward and backward (32*KZ voxels of a column per warp) and
the forward's patch of columns per CTA, per bucket of volume depth and view
count (each rounded up to a power of two), registered in the library as tile
rules (``dgc_bp_add_tile_rule``).  No counterpart in the reference.
"""

from __future__ import annotations

import json
import math
import os
from pathlib import Path

FORWARD_TILES = (8, 4, 2)
BACKWARD_TILES = (8, 4)
TUNE_VIEWS = 48
BP_KZ_FORWARD = (1, 2, 4, 8)
BP_KZ_BACKWARD = (2, 4, 8)
BP_CTAS = ((8, 1), (4, 2))
BP_TUNE_VIEWS = 360
# (arm, slab cells, march unroll, view block): L1 quads unrolled once or twice,
# CTAs in view blocks of 0 (every u tile of a view first), 8, 16, 32 or 64; TMA
# bricks; z pairs through L1
FORWARD_ARMS = ((0, 0, 1, 0), (0, 0, 2, 0), (0, 0, 1, 8), (0, 0, 1, 16), (0, 0, 1, 32),
                (0, 0, 1, 64), (1, 2, 1, 0), (1, 4, 1, 0), (2, 0, 1, 0), (2, 0, 1, 16))
ARM_TUNE_VIEWS = 24


def _pow2(x: float) -> bool:
    m, _ = math.frexp(float(x))
    return x > 0 and m == 0.5


def bucket(problem) -> str:
    """Shape-bucket key of a ``batch.Problem``."""
    D, H, W = (int(s) for s in problem.volume.shape)
    U, V = int(problem.U), int(problem.V)
    vcls = round(math.log2(D * H * W))
    r128 = lambda n: -(-n // 128) * 128  # noqa: E731
    return f"vol2^{vcls}-U{r128(U)}-V{r128(V)}-{'mul' if _pow2(problem.voxel_size) else 'div'}"


def default_cache_path() -> Path:
    env = os.environ.get("DGC_TUNE_CACHE")
    if env:
        return Path(env)
    return Path.home() / ".cache" / "dgc_b200" / "tiles.json"


def time_problem(problem, direction: str, tile: int, grad_volume=True, warmup=1, repeats=3):
    """Median device time [ms] of one forward or backward launch of ``problem``
    restricted to its first ``TUNE_VIEWS`` views."""
    import torch

    from .batch import ProjectionBatch, Problem

    tiles = (tile, 8) if direction == "forward" else (8, tile)
    views = min(int(problem.geometry[0].numel()), TUNE_VIEWS)
    pr = Problem(**{**problem.__dict__, "tiles": tiles, "grad_projections": None,
                    "geometry": [g[:views] for g in problem.geometry]})
    batch = ProjectionBatch([pr], grad_volume=grad_volume)
    batch.forward()
    run = batch.forward if direction == "forward" else (lambda: batch.backward(False))
    for _ in range(warmup):
        run()
    times = []
    for _ in range(repeats):
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        run()
        stop.record()
        stop.synchronize()
        times.append(start.elapsed_time(stop))
    del batch
    return sorted(times)[len(times) // 2]


def arm_name(arm, slab, unroll, view_block) -> str:
    """Label of a forward arm: l1-unroll1, l1-unroll1-vb64, tma-slab4, pairs, ..."""
    base = {0: f"l1-unroll{unroll}", 1: f"tma-slab{slab}", 2: "pairs"}[int(arm)]
    return base + (f"-vb{view_block}" if view_block else "")


def arm_bucket(volume_shape) -> int:
    """Voxel count of a forward-arm bucket: D*H*W rounded up to a power of two."""
    D, H, W = (int(x) for x in volume_shape)
    return 1 << max(0, (D * H * W - 1).bit_length())


def time_forward_arm(problem, arm, slab, unroll=1, view_block=0, warmup=1, repeats=3):
    """Median device time [ms] of ``project`` of ``problem`` restricted to its
    first ``ARM_TUNE_VIEWS`` views with the forward arm ``arm`` (slab width
    ``slab``, march unroll ``unroll``, CTA view block ``view_block``).  The measurement replaces the library's arm rules by one rule
    for this arm and clears them afterwards (``Autotuner.tune_forward_arm``
    registers its cached rules again)."""
    import torch

    from . import _native, _ops

    views = min(int(problem.geometry[0].numel()), ARM_TUNE_VIEWS)
    geom = [g[:views].contiguous() for g in problem.geometry]
    lib = _native.lib()
    _native.check(lib.dgc_fp_clear_arm_rules())
    _native.check(lib.dgc_fp_add_arm_rule(1 << 62, int(arm), int(slab), int(unroll),
                                          int(view_block)))
    try:
        def run():
            _ops.fp_forward(problem.volume, *geom, problem.pixel_size, problem.U, problem.V,
                            problem.step_size, problem.voxel_size, *problem.offset)
        for _ in range(warmup):
            run()
        times = []
        for _ in range(repeats):
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record()
            run()
            stop.record()
            stop.synchronize()
            times.append(start.elapsed_time(stop))
    finally:
        _native.check(lib.dgc_fp_clear_arm_rules())
    return sorted(times)[len(times) // 2]


def bp_bucket(volume_shape, views):
    """(d_max, a_max) of a backprojection: depth and view count rounded up to powers of two."""
    D, A = int(volume_shape[0]), int(views)
    return 1 << max(0, (D - 1).bit_length()), 1 << max(0, (A - 1).bit_length())


def time_backprojector(projections, geometry, pixel_size, volume_shape, voxel_size,
                       volume_offset, direction, kz, cta=(8, 1), warmup=1, repeats=3):
    """Median device time [ms] of the backprojection (``direction`` "forward")
    or of its backward without the projection gradient ("backward") with Z
    blocking ``kz`` and forward column patch ``cta``, on the first
    ``BP_TUNE_VIEWS`` views.  The measurement replaces the library's tile
    rules by one rule for these tiles and clears the rules afterwards
    (``Autotuner.tune_backprojector`` registers its cached rules again)."""
    import torch

    from . import _native, _ops

    views = min(int(geometry[0].numel()), BP_TUNE_VIEWS)
    proj = projections[:views].contiguous()
    geom = [g[:views].contiguous() for g in geometry]
    D, H, W = (int(x) for x in volume_shape)
    lib = _native.lib()
    _native.check(lib.dgc_bp_clear_tile_rules())
    _native.check(lib.dgc_bp_add_tile_rule(1 << 30, 1 << 30, int(kz), int(kz), int(cta[0]),
                                           int(cta[1])))
    try:
        if direction == "forward":
            def run():
                _ops.bp_forward(proj, *geom, pixel_size, D, H, W, voxel_size, *volume_offset)
        else:
            gv = torch.ones((D, H, W), dtype=torch.float32, device=proj.device)

            def run():
                _ops.bp_backward(gv, proj, *geom, pixel_size, voxel_size, *volume_offset,
                                 compute_grad_proj=False)
        for _ in range(warmup):
            run()
        times = []
        for _ in range(repeats):
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record()
            run()
            stop.record()
            stop.synchronize()
            times.append(start.elapsed_time(stop))
    finally:
        _native.check(lib.dgc_bp_clear_tile_rules())
    return sorted(times)[len(times) // 2]


class Autotuner:
    """Chooses (forward, backward) tiles per shape bucket; caches them as JSON.

    ``measure(problem, direction, tile) -> ms`` defaults to ``time_problem``.
    """

    def __init__(self, cache_path=None, measure=None, grad_volume=True, measure_bp=None,
                 measure_arm=None):
        self.cache_path = Path(cache_path) if cache_path else default_cache_path()
        self.measure = measure or (lambda pr, d, t: time_problem(pr, d, t, grad_volume))
        self.measure_bp = measure_bp or time_backprojector
        self.measure_arm = measure_arm or time_forward_arm
        self.table = {}
        if self.cache_path.exists():
            try:
                self.table = json.loads(self.cache_path.read_text())
            except (OSError, ValueError):
                self.table = {}
        self.measured = []  # buckets measured by this tuner

    def _save(self):
        self.cache_path.parent.mkdir(parents=True, exist_ok=True)
        tmp = self.cache_path.with_suffix(".tmp")
        tmp.write_text(json.dumps(self.table, indent=1, sort_keys=True))
        tmp.replace(self.cache_path)

    def tune_bucket(self, problem):
        key = bucket(problem)
        if key in self.table:
            return self.table[key]
        entry = {}
        for direction, cands in (("forward", FORWARD_TILES), ("backward", BACKWARD_TILES)):
            ms = {str(t): float(self.measure(problem, direction, t)) for t in cands}
            entry[direction] = int(min(ms, key=ms.get))
            entry[direction + "_ms"] = ms
        self.table[key] = entry
        self.measured.append(key)
        self._save()
        return entry

    def tune_backprojector(self, projections, geometry, pixel_size, volume_shape, voxel_size,
                           volume_offset=(0.0, 0.0, 0.0)):
        """Z blocking and column patch of the backprojector for the bucket of
        ``volume_shape`` and the view count; measured once, cached, and
        registered in the library (``apply_backprojector_rules``).

        ``measure_bp(projections, geometry, pixel_size, volume_shape,
        voxel_size, volume_offset, direction, kz, cta) -> ms`` defaults to
        ``time_backprojector``."""
        d_max, a_max = bp_bucket(volume_shape, int(geometry[0].numel()))
        key = f"bp:D{d_max}-A{a_max}"
        if key not in self.table:
            args = (projections, geometry, pixel_size, volume_shape, voxel_size,
                    tuple(float(x) for x in volume_offset))
            fwd = {f"{kz}/{cx}x{cy}": float(self.measure_bp(*args, "forward", kz, (cx, cy)))
                   for kz in BP_KZ_FORWARD for cx, cy in BP_CTAS}
            bwd = {str(kz): float(self.measure_bp(*args, "backward", kz, (8, 1)))
                   for kz in BP_KZ_BACKWARD}
            best = min(fwd, key=fwd.get)
            kz_f, patch = best.split("/")
            cx, cy = (int(x) for x in patch.split("x"))
            self.table[key] = {"d_max": d_max, "a_max": a_max, "kz_forward": int(kz_f),
                               "kz_backward": int(min(bwd, key=bwd.get)), "cta": [cx, cy],
                               "forward_ms": fwd, "backward_ms": bwd}
            self.measured.append(key)
            self._save()
        self.apply_backprojector_rules()
        return self.table[key]

    def tune_forward_arm(self, problem):
        """Arm (L1 quads or TMA bricks) and slab width of the forward projector
        for the volume-size bucket of ``problem``: every arm timed once
        (``measure_arm(problem, arm, slab, unroll, view_block) -> ms``, default
        ``time_forward_arm``), cached, registered (``apply_forward_arm_rules``)."""
        key = f"fp-arm:{arm_bucket(problem.volume.shape)}"
        if key not in self.table:
            ms = {f"{a}/{sl}/{un}/{vb}": float(self.measure_arm(problem, a, sl, un, vb))
                  for a, sl, un, vb in FORWARD_ARMS}
            best = min(ms, key=ms.get)
            a, sl, un, vb = (int(x) for x in best.split("/"))
            self.table[key] = {"voxels_max": arm_bucket(problem.volume.shape), "arm": a,
                               "slab": sl, "unroll": un, "view_block": vb, "ms": ms,
                               "arm_name": arm_name(a, sl, un, vb)}
            self.measured.append(key)
            self._save()
        self.apply_forward_arm_rules()
        return self.table[key]

    def apply_forward_arm_rules(self):
        """Register every cached forward-arm bucket as a library arm rule,
        smallest bucket first."""
        from . import _native

        lib = _native.lib()
        _native.check(lib.dgc_fp_clear_arm_rules())
        rules = sorted((e for k, e in self.table.items() if k.startswith("fp-arm:")),
                       key=lambda e: e["voxels_max"])
        for e in rules[:16]:
            _native.check(lib.dgc_fp_add_arm_rule(int(e["voxels_max"]), int(e["arm"]),
                                                  int(e["slab"]), int(e.get("unroll", 1)),
                                                  int(e.get("view_block", 0))))
        return len(rules[:16])

    def apply_backprojector_rules(self):
        """Register every cached backprojector bucket as a library tile rule,
        tightest bucket first."""
        from . import _native

        lib = _native.lib()
        _native.check(lib.dgc_bp_clear_tile_rules())
        rules = sorted((e for k, e in self.table.items() if k.startswith("bp:")),
                       key=lambda e: (e["d_max"], e["a_max"]))
        for e in rules[:16]:
            _native.check(lib.dgc_bp_add_tile_rule(int(e["d_max"]), int(e["a_max"]),
                                                   int(e["kz_forward"]), int(e["kz_backward"]),
                                                   int(e["cta"][0]), int(e["cta"][1])))
        return len(rules[:16])

    def choose(self, problems):
        """Set ``problem.tiles`` of every problem from its bucket's choice."""
        out = []
        for pr in problems:
            e = self.tune_bucket(pr)
            pr.tiles = (e["forward"], e["backward"])
            out.append(pr.tiles)
        return out


def backprojector_tiles(D, A):
    """(kz_forward, kz_backward, (cta_x, cta_y)) a backprojection of depth D
    over A views uses (dgc_bp_tiles)."""
    import ctypes

    from . import _native

    out = [ctypes.c_int() for _ in range(4)]
    _native.check(_native.lib().dgc_bp_tiles(int(D), int(A), *[ctypes.byref(x) for x in out]))
    return out[0].value, out[1].value, (out[2].value, out[3].value)


__all__ = ["Autotuner", "bucket", "bp_bucket", "arm_bucket", "time_problem",
           "time_backprojector", "time_forward_arm", "arm_name", "backprojector_tiles", "FORWARD_TILES",
           "BACKWARD_TILES", "FORWARD_ARMS"]
