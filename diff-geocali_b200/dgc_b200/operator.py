"""``backproject`` and ``detector_centers`` with a first-order autograd wrapper.

Drop-in for the reference's ``cbct_backprojector/operator.py``
(TomSHINING/diff-geoCali): the same functions, arguments, argument checks
(``TypeError`` / ``ValueError`` under the same conditions) and autograd
behaviour (first order only; a gradient is returned for an input only when it
requires one).  The backprojection and its backward run in ``libdgc.so``.
"""

import math
from numbers import Integral, Real

import torch
from torch.autograd.function import once_differentiable

from . import _ops

_TENSOR_NAMES = ("projections", "angles", "sid", "sod", "det_u0", "det_v0",
                 "src_x", "src_y", "src_z")


def _positive_scalar(value, name):
    """A finite positive Python number as float (operator.py:11-17 of the reference)."""
    if isinstance(value, bool) or not isinstance(value, Real):
        raise TypeError(f"{name} must be a positive Python number")
    value = float(value)
    if not (math.isfinite(value) and value > 0):
        raise ValueError(f"{name} must be finite and positive")
    return value


def _is_int(value):
    return isinstance(value, Integral) and not isinstance(value, bool)


def detector_centers(delta_u, delta_v, detector_u, detector_v, pixel_size):
    """Zero-ray detector centre indices ``((U-1)/2 - du/px, (V-1)/2 - dv/px)``.

    Positive physical offsets decrease the centre index.  Tensor inputs keep
    their autograd history (operator.py:32-45 of the reference).
    """
    pixel_size = _positive_scalar(pixel_size, "pixel_size")
    for name, size in (("detector_u", detector_u), ("detector_v", detector_v)):
        if not _is_int(size) or size < 2:
            raise ValueError(f"{name} must be an integer >= 2")
    centre_u = (detector_u - 1.0) / 2.0
    centre_v = (detector_v - 1.0) / 2.0
    return centre_u - delta_u / pixel_size, centre_v - delta_v / pixel_size


class _Backproject(torch.autograd.Function):
    """Autograd node over the native backprojector (operator.py:48-70 of the reference)."""

    @staticmethod
    def forward(ctx, proj, angles, sid, sod, u0, v0, sx, sy, sz,
                pixel_size, volume_shape, voxel_size, volume_offset):
        inputs = [t.contiguous() for t in (proj, angles, sid, sod, u0, v0, sx, sy, sz)]
        ctx.save_for_backward(*inputs)
        ctx.settings = (pixel_size, voxel_size, tuple(volume_offset))
        return _ops.bp_forward(*inputs, pixel_size, *volume_shape, voxel_size, *volume_offset)

    @staticmethod
    @once_differentiable
    def backward(ctx, grad_volume):
        pixel_size, voxel_size, offset = ctx.settings
        wanted = ctx.needs_input_grad[:9]
        grads = _ops.bp_backward(grad_volume.contiguous(), *ctx.saved_tensors,
                                 pixel_size, voxel_size, *offset, compute_grad_proj=wanted[0])
        return tuple(g if need else None for g, need in zip(grads, wanted)) + (None,) * 4


def backproject(projections, angles, sid, sod, det_u0, det_v0,
                src_x, src_y, src_z, pixel_size, volume_shape, voxel_size,
                volume_offset=(0.0, 0.0, 0.0)):
    """Backproject ``[A,U,V]`` projections into a ``[D,H,W] = [Z,Y,X]`` volume.

    All nine tensors are CUDA float32 on one device; the eight geometry tensors
    have shape ``[A]``.  ``sid`` is the source-detector distance, ``sod`` the
    source-origin distance, angles are radians, detector centres are pixel
    indices and source offsets are world-axis distances.  The result is the
    FDK-weighted sum of bilinear detector samples over views, without
    filtering or angular normalisation; only first derivatives exist.
    ``volume_offset`` is ``(x, y, z)``.
    """
    tensors = (projections, angles, sid, sod, det_u0, det_v0, src_x, src_y, src_z)
    for name, t in zip(_TENSOR_NAMES, tensors):
        if not isinstance(t, torch.Tensor):
            raise TypeError(f"{name} must be a torch.Tensor")
        if t.dtype != torch.float32 or t.device.type != "cuda":
            raise ValueError(f"{name} must be a CUDA float32 tensor")
        if t.device != projections.device:
            raise ValueError("All tensors must be on the same CUDA device")
    if projections.ndim != 3:
        raise ValueError("projections must have shape [A,U,V]")
    num_views, det_u, det_v = projections.shape
    if num_views < 1 or min(det_u, det_v) < 2:
        raise ValueError("projections requires A >= 1 and U,V >= 2")
    for name, t in zip(_TENSOR_NAMES[1:], tensors[1:]):
        if t.shape != (num_views,):
            raise ValueError(f"{name} must have shape [{num_views}]")
    pixel_size = _positive_scalar(pixel_size, "pixel_size")
    voxel_size = _positive_scalar(voxel_size, "voxel_size")
    shape = tuple(volume_shape)
    if len(shape) != 3 or not all(_is_int(s) and s >= 1 for s in shape):
        raise ValueError("volume_shape must contain three positive integers (D,H,W)")
    shape = tuple(int(s) for s in shape)
    if projections.numel() > 2**31 - 1 or math.prod(shape) > 2**31 - 1:
        raise ValueError("Input or volume exceeds the kernel's 32-bit indexing limit")
    if max(shape[:2]) > 8 * 65535:
        raise ValueError("D,H exceed the kernel's 3D CUDA grid limits")
    offset = tuple(volume_offset)
    if len(offset) != 3 or not all(
        isinstance(v, Real) and not isinstance(v, bool) and math.isfinite(v) for v in offset
    ):
        raise ValueError("volume_offset must contain three finite numbers (x,y,z)")
    offset = tuple(float(v) for v in offset)
    return _Backproject.apply(*tensors, pixel_size, shape, voxel_size, offset)
