"""FDK helpers: ``fdk_filter`` and ``reconstruct_fdk``.

Drop-in for the reference's ``cbct_backprojector/filtering.py``
(TomSHINING/diff-geoCali, :54-198) for a uniformly sampled circular scan:
centred cosine preweight (detector/source offsets ignored, as in the
reference), Hann-windowed discrete Ram-Lak filter along U with the
reference's zero padding to 2^bitlen(2U-1), ``pixel_size * sid / sod`` scale,
backprojection, ``pi / A`` normalisation and a clamp at zero.

Differences by design: the filter runs on the GPU as a Toeplitz product (the
exact equivalent of the reference's padded FFT convolution), with a
hand-written backward for the projections and the per-view distances (the
reference gets them from autograd through its torch code), and
``reconstruct_fdk`` filters and backprojects all views in one pass, so
``angle_chunk_size`` is validated but does not split the work.  Inputs must be
CUDA tensors: there is no CPU path.
"""

import math
import operator

import torch
from torch.autograd.function import once_differentiable

from . import _ops


def _check_projections(projections):
    if not isinstance(projections, torch.Tensor):
        raise TypeError("projections must be a torch.Tensor")
    if projections.ndim != 3 or min(projections.shape) < 1:
        raise ValueError("projections must have a nonempty [A, U, V] shape")
    if projections.dtype != torch.float32:
        raise TypeError("projections must have dtype torch.float32")


def _positive_scalar(name, value):
    value = float(value)
    if not (math.isfinite(value) and value > 0):
        raise ValueError(f"{name} must be finite and positive")
    return value


def _check_alpha(alpha):
    alpha = _positive_scalar("alpha", alpha)
    if alpha > 1:
        raise ValueError("alpha must satisfy 0 < alpha <= 1")
    return alpha


def _per_view_distance(name, value, projections):
    """A scalar or one value per view, as a float32 [A] tensor on the projections' device."""
    distance = torch.as_tensor(value, dtype=projections.dtype, device=projections.device)
    distance = distance.reshape(-1)
    views = projections.shape[0]
    if distance.numel() == 1:
        distance = distance.expand(views)
    elif distance.numel() != views:
        raise ValueError(f"{name} must be a scalar or have one value per view")
    if not bool(torch.isfinite(distance).all()) or bool((distance <= 0).any()):
        raise ValueError(f"{name} must contain finite positive distances")
    return distance.contiguous()


class _FdkFilter(torch.autograd.Function):
    """``fdk_filter`` under autograd: gradients for the projections and the
    per-view distances (the reference's torch filter has them from autograd,
    filtering.py:54-104); the backward is ``dgc_fdk_filter_backward``."""

    @staticmethod
    def forward(ctx, projections, sod, sid, pixel_size, alpha):
        out = _ops.fdk_filter(projections, pixel_size, sod, sid, alpha)
        ctx.save_for_backward(projections, sod, sid, out)
        ctx.settings = (pixel_size, alpha)
        return out

    @staticmethod
    @once_differentiable
    def backward(ctx, grad):
        projections, sod, sid, out = ctx.saved_tensors
        pixel_size, alpha = ctx.settings
        need_p, need_sod, need_sid = ctx.needs_input_grad[:3]
        gp, gsod, gsid = _ops.fdk_filter_backward(grad, projections, out, pixel_size, sod, sid,
                                                  alpha, need_projections=need_p,
                                                  need_distances=need_sod or need_sid)
        return (gp if need_p else None, gsod if need_sod else None,
                gsid if need_sid else None, None, None)


def fdk_filter(projections, pixel_size, sod, sid, alpha=0.8):
    """Centred cosine weighting and Hann-windowed discrete ramp filter along U.

    Args:
        projections: CUDA float32 line integrals ``[A, U, V]``.
        pixel_size: detector pixel spacing (same length unit as the distances).
        sod: source-origin distance, scalar or one value per view.
        sid: source-detector distance, scalar or one value per view.
        alpha: Hann cutoff as a fraction of Nyquist, ``0 < alpha <= 1``.

    Returns a contiguous float32 tensor of the same shape, scaled by
    ``pixel_size * sid / sod``.
    """
    _check_projections(projections)
    pixel_size = _positive_scalar("pixel_size", pixel_size)
    alpha = _check_alpha(alpha)
    sod = _per_view_distance("sod", sod, projections)
    sid = _per_view_distance("sid", sid, projections)
    if not projections.is_cuda:
        raise ValueError("fdk_filter requires CUDA projections (there is no CPU path)")
    if torch.is_grad_enabled() and (projections.requires_grad or sod.requires_grad or
                                    sid.requires_grad):
        return _FdkFilter.apply(projections, sod, sid, pixel_size, alpha)
    return _ops.fdk_filter(projections, pixel_size, sod, sid, alpha)


def _fdk_arguments(projections, geometry, pixel_size, volume_shape, voxel_size, volume_offset,
                   alpha, angle_chunk_size):
    """The argument checks of the reference's reconstruct_fdk
    (filtering.py:107-198) on one rank's views; returns (pixel_size,
    volume_shape, voxel_size, offset, alpha)."""
    _check_projections(projections)
    sid, sod = geometry[1], geometry[2]
    if min(projections.shape[1:]) < 2:
        raise ValueError("reconstruct_fdk requires detector dimensions U and V >= 2")
    views = projections.shape[0]
    names = ("angles", "sid", "sod", "det_u0", "det_v0", "src_x", "src_y", "src_z")
    for name, t in zip(names, geometry):
        if not isinstance(t, torch.Tensor):
            raise TypeError(f"{name} must be a torch.Tensor of shape [A]")
        if t.ndim != 1 or t.numel() != views:
            raise ValueError(f"{name} must have shape [{views}]")
        if t.dtype != projections.dtype or t.device != projections.device:
            raise ValueError(f"{name} must match the projections' dtype and device")
    if not bool(torch.isfinite(torch.stack(geometry)).all()):
        raise ValueError("geometry must contain only finite values")
    if bool((sid <= 0).any()) or bool((sod <= 0).any()):
        raise ValueError("sid and sod must contain positive distances")
    pixel_size = _positive_scalar("pixel_size", pixel_size)
    voxel_size = _positive_scalar("voxel_size", voxel_size)
    alpha = _check_alpha(alpha)
    try:
        angle_chunk_size = operator.index(angle_chunk_size)
        volume_shape = tuple(operator.index(s) for s in volume_shape)
    except TypeError as error:
        raise TypeError("angle_chunk_size and volume dimensions must be integers") from error
    if angle_chunk_size < 1:
        raise ValueError("angle_chunk_size must be at least 1")
    if len(volume_shape) != 3 or min(volume_shape) < 1:
        raise ValueError("volume_shape must contain three positive dimensions (D, H, W)")
    if math.prod(volume_shape) > 2**31 - 1:
        raise ValueError("volume exceeds the backprojector's 32-bit indexing limit")
    if max(volume_shape[:2]) > 8 * 65535:
        raise ValueError("D,H exceed the backprojector's 3D CUDA grid limits")
    if min(views, angle_chunk_size) * math.prod(projections.shape[1:]) > 2**31 - 1:
        raise ValueError("Reduce angle_chunk_size to fit the backprojector's 32-bit indexing limit")
    offset = tuple(float(v) for v in volume_offset)
    if len(offset) != 3 or not all(math.isfinite(v) for v in offset):
        raise ValueError("volume_offset must contain three finite values")
    return pixel_size, volume_shape, voxel_size, offset, alpha


@torch.no_grad()
def reconstruct_fdk(
    projections,
    angles,
    sid,
    sod,
    det_u0,
    det_v0,
    src_x,
    src_y,
    src_z,
    pixel_size,
    volume_shape,
    voxel_size,
    volume_offset=(0.0, 0.0, 0.0),
    alpha=0.8,
    angle_chunk_size=32,
    short_scan=False,
):
    """FDK reconstruction: filter, backproject, multiply by ``pi / A``, clamp at 0.

    ``projections`` is CUDA float32 ``[A, U, V]``; ``angles`` .. ``src_z`` are
    float32 ``[A]`` tensors on the same device (radians, pixel-index detector
    centres).  ``volume_shape`` is ``(D, H, W)``; ``volume_offset`` follows
    ``backproject``.  Uniform angular weights assume a complete, uniformly
    sampled circular scan; the cosine preweight is centred.

    ``short_scan=True`` (an addition to the reference's signature) treats the
    views as a uniformly spaced short scan over ``angles[0] .. angles[-1]``
    (monotone, covering pi plus twice the largest fan angle): Parker weights
    multiply the cosine preweight and the view spacing replaces ``pi / A``.
    """
    _check_projections(projections)
    if not projections.is_cuda:
        raise ValueError("reconstruct_fdk requires CUDA projections")
    geometry = (angles, sid, sod, det_u0, det_v0, src_x, src_y, src_z)
    pixel_size, volume_shape, voxel_size, offset, alpha = _fdk_arguments(
        projections, geometry, pixel_size, volume_shape, voxel_size, volume_offset, alpha,
        angle_chunk_size)
    views = projections.shape[0]
    if short_scan:
        a0, a1 = float(angles[0]), float(angles[-1])
        span = abs(a1 - a0)
        fan = math.atan(((projections.shape[1] - 1) / 2 * pixel_size) / float(sid.min()))
        if views < 2 or span < math.pi + 2 * fan - 1e-6:
            raise ValueError("a short scan must cover pi plus twice the largest fan angle "
                             f"({math.degrees(math.pi + 2 * fan):.2f} deg); got "
                             f"{math.degrees(span):.2f} deg")
        steps = torch.diff(angles.double()) * (1.0 if a1 >= a0 else -1.0)
        if bool((steps <= 0).any()):
            raise ValueError("short-scan angles must be strictly monotone")
        weights = _ops.parker_weights(angles, sid, projections.shape[1], pixel_size)
        return _ops.reconstruct_fdk_weighted(projections, geometry, pixel_size, volume_shape,
                                             voxel_size, offset, alpha, weights,
                                             span / (views - 1))
    return _ops.reconstruct_fdk(projections, geometry, pixel_size, volume_shape, voxel_size,
                                offset, alpha)
