"""``project``: differentiable source-only cone-beam ray integrator.

Drop-in for the reference's ``cbct_backprojector/source_only_forward_projector.py``
(TomSHINING/diff-geoCali): same arguments, the same argument checks
(``TypeError`` / ``ValueError`` under the same conditions, :30-71), the same
autograd Function (first order, optional ROI arguments for direct
``apply`` callers, gradients only where requested, :75-116).  The ray march
and its backward run in ``libdgc.so``.
"""

import math
from numbers import Integral, Real

import torch
from torch.autograd import Function

from . import _ops
from .operator import _positive_scalar

_TENSOR_NAMES = ("volume", "angles", "sid", "sod", "det_u0_arr", "det_v0_arr",
                 "src_x_arr", "src_y_arr", "src_z_arr")


def _validate_inputs(volume, angles, sid, sod, det_u0_arr, det_v0_arr,
                     src_x_arr, src_y_arr, src_z_arr, pixel_size,
                     detector_u, detector_v, step_size, voxel_size,
                     off_x, off_y, off_z):
    tensors = (volume, angles, sid, sod, det_u0_arr, det_v0_arr, src_x_arr, src_y_arr, src_z_arr)
    for name, t in zip(_TENSOR_NAMES, tensors):
        if not isinstance(t, torch.Tensor):
            raise TypeError(f"{name} must be a torch.Tensor")
        if t.dtype != torch.float32 or t.device.type != "cuda":
            raise ValueError(f"{name} must be a CUDA float32 tensor")
        if t.device != volume.device:
            raise ValueError("All tensors must be on the same CUDA device")
    if volume.ndim != 3 or min(volume.shape) < 1:
        raise ValueError("volume must have a nonempty [D,H,W] shape")
    if angles.ndim != 1 or angles.numel() < 1:
        raise ValueError("angles must have a nonempty shape [A]")
    num_views = angles.numel()
    for name, t in zip(_TENSOR_NAMES[1:], tensors[1:]):
        if t.shape != (num_views,):
            raise ValueError(f"{name} must have shape [{num_views}]")
    for name, size in (("detector_u", detector_u), ("detector_v", detector_v)):
        if isinstance(size, bool) or not isinstance(size, Integral):
            raise TypeError(f"{name} must be a positive integer")
        if size < 1:
            raise ValueError(f"{name} must be a positive integer")
    offsets = (off_x, off_y, off_z)
    for name, value in zip(("off_x", "off_y", "off_z"), offsets):
        if isinstance(value, bool) or not isinstance(value, Real):
            raise TypeError(f"{name} must be a finite Python number")
        if not math.isfinite(value):
            raise ValueError(f"{name} must be finite")
    return (
        _positive_scalar(pixel_size, "pixel_size"),
        int(detector_u),
        int(detector_v),
        _positive_scalar(step_size, "step_size"),
        _positive_scalar(voxel_size, "voxel_size"),
        *(float(v) for v in offsets),
    )


class DifferentiableSourceOnlyForwardProjector(Function):
    """Autograd node over the native forward projector."""

    @staticmethod
    def forward(ctx, volume, angles, sid, sod, det_u0_arr, det_v0_arr,
                src_x_arr, src_y_arr, src_z_arr, pixel_size,
                detector_u, detector_v, step_size, voxel_size,
                off_x=0.0, off_y=0.0, off_z=0.0):
        (pixel_size, detector_u, detector_v, step_size, voxel_size,
         off_x, off_y, off_z) = _validate_inputs(
            volume, angles, sid, sod, det_u0_arr, det_v0_arr, src_x_arr, src_y_arr, src_z_arr,
            pixel_size, detector_u, detector_v, step_size, voxel_size, off_x, off_y, off_z)
        inputs = [t.contiguous() for t in (volume, angles, sid, sod, det_u0_arr, det_v0_arr,
                                           src_x_arr, src_y_arr, src_z_arr)]
        ctx.save_for_backward(*inputs)
        ctx.settings = (pixel_size, step_size, voxel_size, off_x, off_y, off_z)
        # Direct apply(...) callers may leave out the three ROI offsets.
        ctx.num_inputs = len(ctx.needs_input_grad)
        return _ops.fp_forward(*inputs, pixel_size, detector_u, detector_v, step_size, voxel_size,
                               off_x, off_y, off_z)

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, grad_projection):
        pixel_size, step_size, voxel_size, off_x, off_y, off_z = ctx.settings
        wanted = ctx.needs_input_grad[:9]
        grads = _ops.fp_backward(grad_projection.contiguous(), *ctx.saved_tensors,
                                 pixel_size, step_size, voxel_size, bool(wanted[0]),
                                 off_x, off_y, off_z)
        result = tuple(g if need else None for g, need in zip(grads, wanted)) + (None,) * 8
        return result[:ctx.num_inputs]


def project(volume, angles, sid, sod, det_u0_arr, det_v0_arr,
            src_x_arr, src_y_arr, src_z_arr, pixel_size,
            detector_u, detector_v, step_size=0.2, voxel_size=1.0,
            off_x=0.0, off_y=0.0, off_z=0.0):
    """Physical ray-integral projections with layout ``[A,U,V]``.

    ``volume`` is CUDA float32 ``[D,H,W]``; the eight geometry tensors are CUDA
    float32 ``[A]`` on the same device.  ``sid`` is the source-detector
    distance; source offsets are world-coordinate and move only the source; the
    detector stays at local y = sod - sid.  Voxel ``x`` sits at
    ``(x - W/2) * voxel_size + off_x`` (likewise y, z).  The integrator
    samples the trilinear volume at fixed steps from the box entry; its
    first-order gradients are piecewise (sample-count, cell and entry-face
    changes are not differentiated).  Scalar settings have no gradients.
    """
    return DifferentiableSourceOnlyForwardProjector.apply(
        volume, angles, sid, sod, det_u0_arr, det_v0_arr,
        src_x_arr, src_y_arr, src_z_arr, pixel_size,
        detector_u, detector_v, step_size, voxel_size,
        off_x, off_y, off_z,
    )
