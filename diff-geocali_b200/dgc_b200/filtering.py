"""FDK helpers: ``fdk_filter`` and ``reconstruct_fdk``.

Drop-in for the reference's ``cbct_backprojector/filtering.py``
(TomSHINING/diff-geoCali, :54-198) for a uniformly sampled circular scan:
centred cosine preweight (detector/source offsets ignored, as in the
reference), Hann-windowed discrete Ram-Lak filter along U with the
reference's zero padding to 2^bitlen(2U-1), ``pixel_size * sid / sod`` scale,
backprojection, ``pi / A`` normalisation and a clamp at zero.

Additions beyond the reference's signatures, off by default: Parker-weighted
short scans (``reconstruct_fdk(short_scan=True)``) and an offset-aware cosine
preweight (``fdk_filter(frame=...)``, ``reconstruct_fdk(offset_preweight=True)``,
``preweight_frame``).

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


def _per_view_value(name, value, projections):
    """A finite scalar or one value per view, as a float32 [A] tensor on the projections' device."""
    values = torch.as_tensor(value, dtype=projections.dtype, device=projections.device)
    values = values.reshape(-1)
    views = projections.shape[0]
    if values.numel() == 1:
        values = values.expand(views)
    elif values.numel() != views:
        raise ValueError(f"{name} must be a scalar or have one value per view")
    if not bool(torch.isfinite(values).all()):
        raise ValueError(f"{name} must contain finite values")
    return values.contiguous()


def _check_frame(frame, projections):
    """``frame = (dist, u, v)`` with None entries as float32 [A] tensors (or None)."""
    if frame is None:
        return (None, None, None)
    if not isinstance(frame, (tuple, list)) or len(frame) != 3:
        raise TypeError("frame must be a (dist, u, v) triple")
    dist, u, v = frame
    return (None if dist is None else _per_view_distance("frame dist", dist, projections),
            None if u is None else _per_view_value("frame u", u, projections),
            None if v is None else _per_view_value("frame v", v, projections))


def preweight_frame(angles, sid, sod, det_u0, det_v0, src_x, src_y, src_z, pixel_size):
    """The cosine preweight's frame of each view from the scan geometry (the
    eight per-view arrays in the operators' order; ``sod`` does not enter),
    as differentiable torch ops: ``(dist, u, v)`` with ``dist = sid + ds_n``
    the source's distance to the detector plane and ``(u, v) = (det_u0 +
    ds_u / pixel_size, det_v0 + src_z / pixel_size)`` the pixel indices where
    the perpendicular from the source meets the detector, ``ds_u`` and
    ``ds_n`` the source offset along the detector's U axis and its normal in
    the rotated system (the backprojector's, bp.cu:53-56).  With zero source
    offsets and centred detectors it is the reference's centred weight
    (filtering.py:82-85)."""
    pixel_size = _positive_scalar("pixel_size", pixel_size)
    c, s = torch.cos(angles), torch.sin(angles)
    ds_u = src_x * c + src_y * s
    ds_n = -src_x * s + src_y * c
    return sid + ds_n, det_u0 + ds_u / pixel_size, det_v0 + src_z / pixel_size


class _FdkFilter(torch.autograd.Function):
    """``fdk_filter`` under autograd: gradients for the projections, the
    per-view distances and the preweight frame (the reference's torch filter
    has the first two from autograd, filtering.py:54-104); the backward is
    ``dgc_fdk_filter_backward`` (``dgc_fdk_filter_backward_ex`` with a frame)."""

    @staticmethod
    def forward(ctx, projections, sod, sid, dist, fu, fv, pixel_size, alpha):
        frame = (dist, fu, fv)
        ctx.framed = any(t is not None for t in frame)
        if ctx.framed:
            out = _ops.fdk_filter_framed(projections, pixel_size, sod, sid, alpha, frame)
        else:
            out = _ops.fdk_filter(projections, pixel_size, sod, sid, alpha)
        ctx.save_for_backward(projections, sod, sid, out, dist, fu, fv)
        ctx.settings = (pixel_size, alpha)
        return out

    @staticmethod
    @once_differentiable
    def backward(ctx, grad):
        projections, sod, sid, out, dist, fu, fv = ctx.saved_tensors
        pixel_size, alpha = ctx.settings
        need = ctx.needs_input_grad
        if ctx.framed:
            grads = _ops.fdk_filter_backward_framed(grad, projections, out, pixel_size, sod, sid,
                                                    alpha, (dist, fu, fv), need[0], need[1],
                                                    need[2], need[3:6])
        else:
            grads = _ops.fdk_filter_backward(grad, projections, out, pixel_size, sod, sid, alpha,
                                             need_projections=need[0],
                                             need_distances=need[1] or need[2])
            grads = (*grads, None, None, None)
        return (*(g if n else None for g, n in zip(grads, need[:6])), None, None)


def fdk_filter(projections, pixel_size, sod, sid, alpha=0.8, *, frame=None):
    """Cosine weighting and Hann-windowed discrete ramp filter along U.

    Args:
        projections: CUDA float32 line integrals ``[A, U, V]``.
        pixel_size: detector pixel spacing (same length unit as the distances).
        sod: source-origin distance, scalar or one value per view.
        sid: source-detector distance, scalar or one value per view.
        alpha: Hann cutoff as a fraction of Nyquist, ``0 < alpha <= 1``.
        frame: (an addition to the reference's signature) ``(dist, u, v)``,
            each None, a scalar or one value per view: the cosine preweight is
            ``dist / sqrt(dist^2 + ((i - u) px)^2 + ((j - v) px)^2)`` at pixel
            ``(i, j)``, i.e. taken from a source at distance ``dist`` from the
            detector plane whose perpendicular meets it at pixel ``(u, v)``
            (``preweight_frame`` builds it from the geometry).  None entries
            keep the reference's centred weight (sid, (U-1)/2, (V-1)/2).
            Differentiable in each entry.

    Returns a contiguous float32 tensor of the same shape, scaled by
    ``pixel_size * sid / sod``.
    """
    _check_projections(projections)
    pixel_size = _positive_scalar("pixel_size", pixel_size)
    alpha = _check_alpha(alpha)
    sod = _per_view_distance("sod", sod, projections)
    sid = _per_view_distance("sid", sid, projections)
    frame = _check_frame(frame, projections)
    if not projections.is_cuda:
        raise ValueError("fdk_filter requires CUDA projections (there is no CPU path)")
    framed = any(t is not None for t in frame)
    if torch.is_grad_enabled() and any(t is not None and t.requires_grad
                                       for t in (projections, sod, sid, *frame)):
        return _FdkFilter.apply(projections, sod, sid, *frame, pixel_size, alpha)
    if framed:
        return _ops.fdk_filter_framed(projections, pixel_size, sod, sid, alpha, frame)
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
    offset_preweight=False,
):
    """FDK reconstruction: filter, backproject, multiply by ``pi / A``, clamp at 0.

    ``projections`` is CUDA float32 ``[A, U, V]``; ``angles`` .. ``src_z`` are
    float32 ``[A]`` tensors on the same device (radians, pixel-index detector
    centres).  ``volume_shape`` is ``(D, H, W)``; ``volume_offset`` follows
    ``backproject``.  Uniform angular weights assume a complete, uniformly
    sampled circular scan; the cosine preweight is centred unless
    ``offset_preweight`` is set.

    ``short_scan=True`` (an addition to the reference's signature) treats the
    views as a uniformly spaced short scan over ``angles[0] .. angles[-1]``
    (monotone, covering pi plus twice the largest fan angle): Parker weights
    multiply the cosine preweight and the view spacing replaces ``pi / A``.

    ``offset_preweight=True`` (also an addition) takes the cosine preweight,
    and the Parker fan angles, in each view's ``preweight_frame``: the cosine
    of each ray's angle to the detector normal from the actual source
    position, where the reference centres it on the detector array whatever
    the detector and source offsets (filtering.py:1-8, 70-71).
    """
    _check_projections(projections)
    if not projections.is_cuda:
        raise ValueError("reconstruct_fdk requires CUDA projections")
    geometry = (angles, sid, sod, det_u0, det_v0, src_x, src_y, src_z)
    pixel_size, volume_shape, voxel_size, offset, alpha = _fdk_arguments(
        projections, geometry, pixel_size, volume_shape, voxel_size, volume_offset, alpha,
        angle_chunk_size)
    views = projections.shape[0]
    frame = None
    if offset_preweight:
        frame = preweight_frame(*geometry, pixel_size)
        if bool((frame[0] <= 0).any()):
            raise ValueError("the source must lie in front of the detector plane")
    U = projections.shape[1]
    if short_scan:
        a0, a1 = float(angles[0]), float(angles[-1])
        span = abs(a1 - a0)
        if frame is None:
            fan = math.atan(((U - 1) / 2 * pixel_size) / float(sid.min()))
        else:
            reach = torch.maximum(frame[1], (U - 1) - frame[1]) * pixel_size
            fan = float(torch.atan(reach / frame[0]).max())
        if views < 2 or span < math.pi + 2 * fan - 1e-6:
            raise ValueError("a short scan must cover pi plus twice the largest fan angle "
                             f"({math.degrees(math.pi + 2 * fan):.2f} deg); got "
                             f"{math.degrees(span):.2f} deg")
        steps = torch.diff(angles.double()) * (1.0 if a1 >= a0 else -1.0)
        if bool((steps <= 0).any()):
            raise ValueError("short-scan angles must be strictly monotone")
        if frame is None:
            weights = _ops.parker_weights(angles, sid, U, pixel_size)
            return _ops.reconstruct_fdk_weighted(projections, geometry, pixel_size, volume_shape,
                                                 voxel_size, offset, alpha, weights,
                                                 span / (views - 1))
        weights = _ops.parker_weights(angles, sid, U, pixel_size, frame[0], frame[1])
        return _ops.reconstruct_fdk_ex(projections, geometry, pixel_size, volume_shape,
                                       voxel_size, offset, alpha, frame, weights,
                                       span / (views - 1))
    if frame is not None:
        return _ops.reconstruct_fdk_ex(projections, geometry, pixel_size, volume_shape,
                                       voxel_size, offset, alpha, frame, None, math.pi / views)
    return _ops.reconstruct_fdk(projections, geometry, pixel_size, volume_shape, voxel_size,
                                offset, alpha)
