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
first ``TUNE_VIEWS`` views.  No counterpart in the reference.
"""

from __future__ import annotations

import json
import math
import os
from pathlib import Path

FORWARD_TILES = (8, 4, 2)
BACKWARD_TILES = (8, 4)
TUNE_VIEWS = 48


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


class Autotuner:
    """Chooses (forward, backward) tiles per shape bucket; caches them as JSON.

    ``measure(problem, direction, tile) -> ms`` defaults to ``time_problem``.
    """

    def __init__(self, cache_path=None, measure=None, grad_volume=True):
        self.cache_path = Path(cache_path) if cache_path else default_cache_path()
        self.measure = measure or (lambda pr, d, t: time_problem(pr, d, t, grad_volume))
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

    def choose(self, problems):
        """Set ``problem.tiles`` of every problem from its bucket's choice."""
        out = []
        for pr in problems:
            e = self.tune_bucket(pr)
            pr.tiles = (e["forward"], e["backward"])
            out.append(pr.tiles)
        return out


__all__ = ["Autotuner", "bucket", "time_problem", "FORWARD_TILES", "BACKWARD_TILES"]
