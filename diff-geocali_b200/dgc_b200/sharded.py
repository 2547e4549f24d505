"""View-sharded operators: one scan split across ranks (one process per GPU).

Every operator here treats the views of a scan independently, so a scan is
split into contiguous view ranges, one per rank (``view_shard``), and each rank
holds only its views' projections and geometry:

* ``reconstruct_fdk_sharded`` -- each rank filters and backprojects its views
  into an unclamped partial volume (``dgc_reconstruct_fdk_partial``, angular
  factor pi / views of the whole scan), one all-reduce sums the partial
  volumes (NCCL over NVLink for CUDA tensors) and every rank clamps the sum
  (``dgc_clamp_volume``).  The result is ``reconstruct_fdk`` of the whole scan
  up to the order of the float additions.
* ``backproject_sharded`` -- ``backproject`` summed over the ranks' views
  under autograd: the forward all-reduces the partial volumes; the backward is
  local, because every rank holds the same gradient of the replicated volume.
* ``project_sharded`` -- ``project`` of a replicated volume onto this rank's
  views: nothing is exchanged in the forward; the backward all-reduces the
  volume gradient (the adjoint summed over all views), while the geometry
  gradients stay with the views they belong to.
* ``calibrate_sharded`` -- per-view geometry calibration of the rank's views
  (the offsets of different views never interact); only the loss
  normalisation and the stopping metrics are summed over the ranks.
* ``reconstruct_fdk_slab`` -- the other split: every rank holds all views and
  reconstructs only its slab of depth rows (``slab_shard``), a sub-volume
  whose ``volume_offset`` puts its voxels where the whole volume's are.
  Nothing is exchanged (``gather_slabs`` assembles the volume when a caller
  wants it whole), each rank holds 1/N of the volume, and short scans work
  (each rank sees the whole scan).

The exchange is one volume per call (67 MB at 256^3) after all of a rank's
compute, so it is a single collective rather than a compute kernel fused with
peer-memory transfers.  Without an initialised process group the functions
are the single-device operators (with one, the all-reduces run whatever its
size).  The reference runs
on one device (filtering.py:107-198, operator.py:73-127,
source_only_forward_projector.py:119-145); no counterpart there.
"""

from __future__ import annotations

import math

import torch
import torch.distributed as dist

from . import _ops
from .filtering import _fdk_arguments, preweight_frame
from .operator import backproject
from .source_only_forward_projector import project


def view_shard(views, world_size, rank):
    """The contiguous view range ``range(start, stop)`` of ``rank``: balanced,
    the first ``views % world_size`` ranks take one view more."""
    views, world_size, rank = int(views), int(world_size), int(rank)
    if views < 0 or world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("need views >= 0, world_size >= 1 and 0 <= rank < world_size")
    base, extra = divmod(views, world_size)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def _all_reduce_sum(tensor, group=None):
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(tensor, op=dist.ReduceOp.SUM, group=group)
    return tensor


def total_views(local_views, device, group=None):
    """Views of the whole scan: the sum of every rank's view count."""
    n = torch.tensor([int(local_views)], dtype=torch.int64, device=device)
    return int(_all_reduce_sum(n, group).item())


class _SumAcrossRanks(torch.autograd.Function):
    """Forward: the sum of ``x`` over the ranks.  Backward: the gradient as it
    is (the summed tensor is replicated, so every rank holds its gradient)."""

    @staticmethod
    def forward(ctx, x, group):
        return _all_reduce_sum(x.clone(), group)

    @staticmethod
    def backward(ctx, grad):
        return grad, None


class _SumGradAcrossRanks(torch.autograd.Function):
    """Forward: ``x`` as it is (a replicated input).  Backward: the gradient
    summed over the ranks (each rank's share of the uses of ``x``)."""

    @staticmethod
    def forward(ctx, x, group):
        ctx.group = group
        return x.view_as(x)

    @staticmethod
    def backward(ctx, grad):
        return _all_reduce_sum(grad.contiguous().clone(), ctx.group), None


def _partial_volume(projections, geometry, pixel_size, volume_shape, voxel_size, offset, alpha,
                    angle_scale, frame=None):
    if not projections.is_cuda:
        raise ValueError("reconstruct_fdk_sharded requires CUDA projections")
    if frame is None:
        return _ops.reconstruct_fdk_partial(projections, geometry, pixel_size, volume_shape,
                                            voxel_size, offset, alpha, None, angle_scale)
    return _ops.reconstruct_fdk_ex(projections, geometry, pixel_size, volume_shape, voxel_size,
                                   offset, alpha, frame, None, angle_scale, clamp=False)


def _clamp(volume):
    return _ops.clamp_volume(volume)


@torch.no_grad()
def reconstruct_fdk_sharded(projections, angles, sid, sod, det_u0, det_v0, src_x, src_y, src_z,
                            pixel_size, volume_shape, voxel_size, volume_offset=(0.0, 0.0, 0.0),
                            alpha=0.8, angle_chunk_size=32, views_total=None, group=None,
                            offset_preweight=False):
    """``reconstruct_fdk`` of a full circular scan whose views are spread over
    the ranks of ``group``; every rank passes its own views (``[A_r, U, V]``
    projections and ``[A_r]`` geometry) and receives the whole volume.

    ``views_total`` (the scan's view count) is summed over the ranks when
    omitted.  ``offset_preweight`` is ``reconstruct_fdk``'s (the frames are
    per view, so each rank computes its own).  Argument checks and errors are
    those of ``reconstruct_fdk`` on the rank's views.
    """
    geometry = (angles, sid, sod, det_u0, det_v0, src_x, src_y, src_z)
    pixel_size, volume_shape, voxel_size, offset, alpha = _fdk_arguments(
        projections, geometry, pixel_size, volume_shape, voxel_size, volume_offset, alpha,
        angle_chunk_size)
    if views_total is None:
        views_total = total_views(projections.shape[0], projections.device, group)
    if int(views_total) < projections.shape[0]:
        raise ValueError("views_total must count the views of every rank")
    frame = None
    if offset_preweight:
        frame = preweight_frame(*geometry, pixel_size)
        if bool((frame[0] <= 0).any()):
            raise ValueError("the source must lie in front of the detector plane")
    volume = _partial_volume(projections, geometry, pixel_size, volume_shape, voxel_size, offset,
                             alpha, math.pi / int(views_total), frame)
    _all_reduce_sum(volume, group)
    return _clamp(volume)


def backproject_sharded(projections, angles, sid, sod, det_u0, det_v0, src_x, src_y, src_z,
                        pixel_size, volume_shape, voxel_size, volume_offset=(0.0, 0.0, 0.0),
                        group=None):
    """``backproject`` of this rank's views, summed over the ranks of ``group``
    (differentiable; arguments as ``backproject``)."""
    partial = backproject(projections, angles, sid, sod, det_u0, det_v0, src_x, src_y, src_z,
                          pixel_size, volume_shape, voxel_size, volume_offset)
    return _SumAcrossRanks.apply(partial, group)


def project_sharded(volume, angles, sid, sod, det_u0_arr, det_v0_arr, src_x_arr, src_y_arr,
                    src_z_arr, pixel_size, detector_u, detector_v, step_size=0.2, voxel_size=1.0,
                    off_x=0.0, off_y=0.0, off_z=0.0, group=None):
    """``project`` of a volume replicated on every rank of ``group`` onto this
    rank's views (arguments as ``project``); the volume's gradient is summed
    over the ranks."""
    shared = _SumGradAcrossRanks.apply(volume, group) if volume.requires_grad else volume
    return project(shared, angles, sid, sod, det_u0_arr, det_v0_arr, src_x_arr, src_y_arr,
                   src_z_arr, pixel_size, detector_u, detector_v, step_size, voxel_size, off_x,
                   off_y, off_z)


def calibrate_sharded(volume, measured, nominal, scan, group=None, **kwargs):
    """``calibration.calibrate`` of one scan whose views are spread over the
    ranks of ``group``: every rank passes the replicated volume and its own
    views' ``measured`` / ``mask`` / ``nominal`` / ``warm_start`` /
    ``true_geometry`` and gets its views' offsets.  The per-view offsets are
    independent, so nothing is exchanged per step but the loss normalisation
    (once), the recorded loss and the stopping metrics (a few FP64 numbers per
    iteration); each rank's result equals one calibration over all views,
    restricted to its views."""
    from .calibration import calibrate

    return calibrate(volume, measured, nominal, scan,
                     reduce=lambda t: _all_reduce_sum(t.contiguous().clone(), group), **kwargs)


def slab_shard(depth, world_size, rank):
    """The contiguous range of depth rows (z indices) of ``rank``: balanced as
    ``view_shard``."""
    return view_shard(depth, world_size, rank)


def slab_offset(volume_shape, voxel_size, volume_offset, rows):
    """``volume_offset`` of the sub-volume made of depth rows ``rows`` (a
    range) of a ``volume_shape`` volume, so that its voxel centres are the
    whole volume's: the centre of depth row z is ``(z - D/2) * voxel +
    off_z`` (bp.cu:37-39), so the slab's is ``off_z + (start + d/2 - D/2) *
    voxel`` for ``d`` rows from ``start``."""
    D = int(volume_shape[0])
    d = len(rows)
    ox, oy, oz = (float(v) for v in volume_offset)
    return (ox, oy, oz + (rows.start + d / 2 - D / 2) * float(voxel_size))


def _world(group):
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(group), dist.get_rank(group)
    return 1, 0


def reconstruct_fdk_slab(projections, angles, sid, sod, det_u0, det_v0, src_x, src_y, src_z,
                         pixel_size, volume_shape, voxel_size, volume_offset=(0.0, 0.0, 0.0),
                         alpha=0.8, angle_chunk_size=32, short_scan=False,
                         offset_preweight=False, group=None):
    """This rank's slab of ``reconstruct_fdk`` of the whole scan: every rank
    passes all views and gets ``(slab, rows)``, ``slab`` the ``[len(rows), H,
    W]`` depth rows ``rows = slab_shard(D, world, rank)`` of the volume (up to
    the float rounding of the voxel centres).  No collective.  Without a
    process group it is the whole volume.  Arguments as ``reconstruct_fdk``."""
    from .filtering import reconstruct_fdk

    world, rank = _world(group)
    shape = tuple(int(n) for n in volume_shape)
    if len(shape) != 3:
        raise ValueError("volume_shape must contain three positive dimensions (D, H, W)")
    rows = slab_shard(shape[0], world, rank)
    if len(rows) == 0:
        return projections.new_empty((0, shape[1], shape[2])), rows
    slab = reconstruct_fdk(projections, angles, sid, sod, det_u0, det_v0, src_x, src_y, src_z,
                           pixel_size, (len(rows), shape[1], shape[2]), voxel_size,
                           volume_offset=slab_offset(shape, voxel_size, volume_offset, rows),
                           alpha=alpha, angle_chunk_size=angle_chunk_size, short_scan=short_scan,
                           offset_preweight=offset_preweight)
    return slab, rows


def gather_slabs(slab, depth, group=None):
    """The whole ``[depth, H, W]`` volume on every rank from each rank's
    ``slab_shard`` slab (one all-gather of equal-size padded slabs)."""
    world, _ = _world(group)
    if world == 1:
        return slab
    rows = [slab_shard(depth, world, r) for r in range(world)]
    most = max(len(r) for r in rows)
    pad = slab.new_zeros((most,) + tuple(slab.shape[1:]))
    pad[:slab.shape[0]] = slab
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([part[:len(r)] for part, r in zip(parts, rows)])


__all__ = ["view_shard", "total_views", "reconstruct_fdk_sharded", "backproject_sharded",
           "project_sharded", "calibrate_sharded", "slab_shard", "slab_offset",
           "reconstruct_fdk_slab", "gather_slabs"]
