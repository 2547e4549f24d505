"""Tensor-level operators over ``libdgc`` with the reference's native signatures.

The functions below take and return ``torch.Tensor`` objects exactly like the
reference's pybind11 modules (TomSHINING/diff-geoCali
``csrc/src_cbct_forwardprojector_cuda.cu:732-758`` and
``csrc/src_cbct_backprojector_cuda.cu:524-543``): same argument names and
defaults, same return order, outputs freshly allocated, inputs made
contiguous, launches on the current PyTorch stream of the input's device, no
host synchronisation.  Argument checks raise ``RuntimeError`` with the
reference's messages.  The arithmetic runs in ``libdgc.so`` through the C ABI;
there is no other code path.
"""

from __future__ import annotations

import math

import torch

from . import _native

_GEOM_NAMES = ("angles", "sid", "sod", "det_u0", "det_v0", "src_x", "src_y", "src_z")
_INT_MAX = 2**31 - 1


def _require(cond, msg):
    if not cond:
        raise RuntimeError(msg)


def _workspace(nbytes: int, device) -> torch.Tensor | None:
    if nbytes == 0:
        return None
    return torch.empty(int(nbytes), dtype=torch.uint8, device=device)


def _p(t):
    return None if t is None else t.data_ptr()


def _stream(device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


# ------------------------------------------------------------ forward projector


def _fp_check_geometry(reference, geometry, expected):
    # fp.cu:531-563
    _require(reference.is_cuda, "reference tensor must be CUDA")
    _require(reference.dtype == torch.float32, "reference tensor must be float32")
    for name, t in zip(_GEOM_NAMES, geometry):
        _require(t.is_cuda, f"{name} must be CUDA")
        _require(t.dtype == torch.float32, f"{name} must be float32")
        _require(t.device == reference.device,
                 f"{name} must be on the same CUDA device as the reference tensor")
        _require(t.numel() == expected, f"{name} must contain A elements")


def fp_forward(volume, angles, sid, sod, det_u0_arr, det_v0_arr, src_x_arr, src_y_arr, src_z_arr,
               pixel_size, U, V, step_size, voxel_size, off_x=0.0, off_y=0.0, off_z=0.0):
    """Forward projection [A,U,V] (replaces ``src_cbct_forwardprojector_cuda.forward``)."""
    geometry = (angles, sid, sod, det_u0_arr, det_v0_arr, src_x_arr, src_y_arr, src_z_arr)
    U, V = int(U), int(V)
    pixel_size, step_size, voxel_size = float(pixel_size), float(step_size), float(voxel_size)
    _require(volume.dim() == 3, "volume must have shape [D,H,W]")
    _require(U > 0 and V > 0, "U and V must be positive")
    _require(pixel_size > 0.0 and step_size > 0.0 and voxel_size > 0.0,
             "pixel_size, step_size and voxel_size must be positive")
    A = angles.numel()
    _require(A > 0, "angles must contain at least one view")
    _fp_check_geometry(volume, geometry, A)
    vol = volume.contiguous()
    geom = [t.contiguous() for t in geometry]
    D, H, W = vol.shape
    _require(D > 0 and H > 0 and W > 0, "every volume dimension must be positive")
    out = torch.zeros((A, U, V), dtype=torch.float32, device=vol.device)
    lib = _native.lib()
    with torch.cuda.device(vol.device):
        ws = _workspace(lib.dgc_project_workspace_bytes(D, H, W, A, U, V), vol.device)
        _native.check(lib.dgc_project(
            vol.data_ptr(), D, H, W, *[g.data_ptr() for g in geom], A, pixel_size, U, V,
            step_size, voxel_size, float(off_x), float(off_y), float(off_z), out.data_ptr(),
            _p(ws), 0 if ws is None else ws.numel(), _stream(vol.device)))
    return out


def fp_backward(grad_projection, volume, angles, sid, sod, det_u0_arr, det_v0_arr, src_x_arr,
                src_y_arr, src_z_arr, pixel_size, step_size, voxel_size, compute_grad_volume=True,
                off_x=0.0, off_y=0.0, off_z=0.0):
    """Nine gradients (replaces ``src_cbct_forwardprojector_cuda.backward``)."""
    geometry = (angles, sid, sod, det_u0_arr, det_v0_arr, src_x_arr, src_y_arr, src_z_arr)
    pixel_size, step_size, voxel_size = float(pixel_size), float(step_size), float(voxel_size)
    _require(volume.dim() == 3, "volume must have shape [D,H,W]")
    _require(grad_projection.dim() == 3, "grad_projection must have shape [A,U,V]")
    _require(grad_projection.is_cuda and grad_projection.dtype == torch.float32,
             "grad_projection must be a float32 CUDA tensor")
    _require(grad_projection.device == volume.device,
             "grad_projection and volume must be on the same CUDA device")
    _require(pixel_size > 0.0 and step_size > 0.0 and voxel_size > 0.0,
             "pixel_size, step_size and voxel_size must be positive")
    A, U, V = grad_projection.shape
    _require(A > 0 and U > 0 and V > 0, "every grad_projection dimension must be positive")
    _fp_check_geometry(volume, geometry, A)
    gp = grad_projection.contiguous()
    vol = volume.contiguous()
    geom = [t.contiguous() for t in geometry]
    D, H, W = vol.shape
    _require(D > 0 and H > 0 and W > 0, "every volume dimension must be positive")
    dev = vol.device
    compute = bool(compute_grad_volume)
    grad_volume = torch.zeros_like(vol) if compute else torch.empty(0, dtype=vol.dtype, device=dev)
    grads = [torch.zeros_like(g) for g in geom]
    lib = _native.lib()
    with torch.cuda.device(dev):
        ws = _workspace(lib.dgc_project_backward_workspace_bytes(D, H, W, A, U, V, int(compute)), dev)
        _native.check(lib.dgc_project_backward(
            gp.data_ptr(), vol.data_ptr(), D, H, W, *[g.data_ptr() for g in geom], A, pixel_size,
            U, V, step_size, voxel_size, int(compute), float(off_x), float(off_y), float(off_z),
            grad_volume.data_ptr() if compute else None, *[g.data_ptr() for g in grads],
            _p(ws), 0 if ws is None else ws.numel(), _stream(dev)))
    return [grad_volume, *grads]


def fp_mse_grad(volume, geometry, pixel_size, U, V, step_size, voxel_size, measured, mask=None,
                scale=1.0, offset=(0.0, 0.0, 0.0), return_projection=False):
    """One fused calibration step: ``loss = scale * sum(mask * (p - measured)^2)``
    with ``p = project(volume, geometry)`` and the eight [A] geometry gradients
    of that loss, from one ray march (no volume gradient).  Returns
    ``(loss (0-d float64 tensor), [8 gradients], projection or None)``."""
    pixel_size, step_size, voxel_size = float(pixel_size), float(step_size), float(voxel_size)
    U, V = int(U), int(V)
    _require(volume.dim() == 3, "volume must have shape [D,H,W]")
    A = geometry[0].numel()
    _require(A > 0, "angles must contain at least one view")
    _fp_check_geometry(volume, geometry, A)
    vol = volume.contiguous()
    geom = [t.contiguous() for t in geometry]
    dev = vol.device
    _require(measured.is_cuda and measured.dtype == torch.float32 and measured.device == dev and
             tuple(measured.shape) == (A, U, V), "measured must be float32 [A,U,V] on the volume's device")
    meas = measured.contiguous()
    if mask is not None:
        _require(mask.is_cuda and mask.dtype == torch.float32 and mask.device == dev and
                 tuple(mask.shape) == (A, U, V), "mask must be float32 [A,U,V] on the volume's device")
        mask = mask.contiguous()
    D, H, W = vol.shape
    loss = torch.empty((), dtype=torch.float64, device=dev)
    grads = [torch.empty_like(g) for g in geom]
    proj = torch.empty((A, U, V), dtype=torch.float32, device=dev) if return_projection else None
    lib = _native.lib()
    with torch.cuda.device(dev):
        ws = _workspace(lib.dgc_project_mse_grad_workspace_bytes(D, H, W, A, U, V), dev)
        _native.check(lib.dgc_project_mse_grad(
            vol.data_ptr(), D, H, W, *[g.data_ptr() for g in geom], A, pixel_size, U, V,
            step_size, voxel_size, *(float(x) for x in offset), meas.data_ptr(), _p(mask),
            float(scale), _p(proj), loss.data_ptr(), *[g.data_ptr() for g in grads], _p(ws),
            0 if ws is None else ws.numel(), _stream(dev)))
    return loss, grads, proj


# ---------------------------------------------------------------- backprojector


def _bp_check_projection(proj):
    # bp.cu:298-306
    _require(proj.is_cuda and proj.dtype == torch.float32, "proj must be a CUDA float32 tensor")
    _require(proj.dim() == 3 and proj.size(0) > 0 and proj.size(1) >= 2 and proj.size(2) >= 2,
             "proj must have shape [A,U,V] with A >= 1 and U,V >= 2")
    _require(proj.numel() <= _INT_MAX, "proj exceeds the kernel's 32-bit indexing limit")


def _bp_check_geometry(proj, geometry):
    # bp.cu:308-331
    _bp_check_projection(proj)
    for name, t in zip(_GEOM_NAMES, geometry):
        _require(t.is_cuda and t.dtype == torch.float32 and t.device == proj.device and t.dim() == 1
                 and t.numel() == proj.size(0),
                 f"{name} must be CUDA float32 on proj.device with shape [A]")


def _bp_check_volume_shape(D, H, W):
    # bp.cu:333-341
    _require(0 < D <= _INT_MAX and 0 < H <= _INT_MAX and 0 < W <= _INT_MAX,
             "D,H,W must be positive and fit in a 32-bit integer")
    _require(D * H * W <= _INT_MAX, "volume exceeds the kernel's 32-bit indexing limit")
    _require(D <= 8 * 65535 and H <= 8 * 65535, "D,H exceed the kernel's 3D CUDA grid limits")


def _finite(*values):
    return all(math.isfinite(v) for v in values)


def bp_forward(proj, angles, sid, sod, det_u0_arr, det_v0_arr, src_x_arr, src_y_arr, src_z_arr,
               pixel_size, D, H, W, voxel_size, off_x=0.0, off_y=0.0, off_z=0.0):
    """Backprojection [D,H,W] (replaces ``src_cbct_backprojector_cuda.forward``)."""
    geometry = (angles, sid, sod, det_u0_arr, det_v0_arr, src_x_arr, src_y_arr, src_z_arr)
    pixel_size, voxel_size = float(pixel_size), float(voxel_size)
    off_x, off_y, off_z = float(off_x), float(off_y), float(off_z)
    D, H, W = int(D), int(H), int(W)
    _bp_check_geometry(proj, geometry)
    _bp_check_volume_shape(D, H, W)
    _require(_finite(pixel_size, voxel_size, off_x, off_y, off_z),
             "sizes and ROI offsets must be finite")
    _require(pixel_size > 0.0 and voxel_size > 0.0, "pixel_size and voxel_size must be positive")
    p = proj.contiguous()
    geom = [t.contiguous() for t in geometry]
    A, U, V = p.shape
    dev = p.device
    vol = torch.zeros((D, H, W), dtype=torch.float32, device=dev)
    lib = _native.lib()
    with torch.cuda.device(dev):
        ws = _workspace(lib.dgc_backproject_workspace_bytes(A, U, V, D, H, W), dev)
        _native.check(lib.dgc_backproject(
            p.data_ptr(), A, U, V, *[g.data_ptr() for g in geom], pixel_size, D, H, W, voxel_size,
            off_x, off_y, off_z, vol.data_ptr(), _p(ws), 0 if ws is None else ws.numel(),
            _stream(dev)))
    return vol


def bp_backward(grad_vol, proj, angles, sid, sod, det_u0_arr, det_v0_arr, src_x_arr, src_y_arr,
                src_z_arr, pixel_size, voxel_size, off_x=0.0, off_y=0.0, off_z=0.0,
                compute_grad_proj=True):
    """Nine gradients (replaces ``src_cbct_backprojector_cuda.backward``);
    with ``compute_grad_proj=False`` the first is ``None`` and its scatter is
    skipped."""
    geometry = (angles, sid, sod, det_u0_arr, det_v0_arr, src_x_arr, src_y_arr, src_z_arr)
    pixel_size, voxel_size = float(pixel_size), float(voxel_size)
    off_x, off_y, off_z = float(off_x), float(off_y), float(off_z)
    _bp_check_geometry(proj, geometry)
    _require(grad_vol.is_cuda and grad_vol.dtype == torch.float32 and grad_vol.device == proj.device
             and grad_vol.dim() == 3,
             "grad_vol must be CUDA float32 on proj.device with shape [D,H,W]")
    _bp_check_volume_shape(*grad_vol.shape)
    _require(_finite(pixel_size, voxel_size, off_x, off_y, off_z) and pixel_size > 0.0
             and voxel_size > 0.0,
             "sizes must be finite and positive; ROI offsets must be finite")
    gv = grad_vol.contiguous()
    p = proj.contiguous()
    geom = [t.contiguous() for t in geometry]
    A, U, V = p.shape
    D, H, W = gv.shape
    dev = p.device
    grad_proj = torch.empty_like(p) if compute_grad_proj else None
    grads = [torch.zeros_like(g) for g in geom]
    lib = _native.lib()
    with torch.cuda.device(dev):
        ws = _workspace(lib.dgc_backproject_backward_workspace_bytes(A, U, V, D, H, W), dev)
        _native.check(lib.dgc_backproject_backward(
            gv.data_ptr(), p.data_ptr(), A, U, V, *[g.data_ptr() for g in geom], pixel_size, D, H,
            W, voxel_size, off_x, off_y, off_z, _p(grad_proj),
            *[g.data_ptr() for g in grads], _p(ws), 0 if ws is None else ws.numel(), _stream(dev)))
    return [grad_proj, *grads]


# ------------------------------------------------------------------------- FDK


def fdk_filter(projections, pixel_size, sod, sid, alpha):
    """Cosine-weighted ramp filter along U; ``sod``/``sid`` are CUDA float32 [A]."""
    A, U, V = projections.shape
    p = projections.contiguous()
    dev = p.device
    out = torch.empty_like(p)
    lib = _native.lib()
    with torch.cuda.device(dev):
        ws = _workspace(lib.dgc_fdk_filter_workspace_bytes(A, U, V), dev)
        _native.check(lib.dgc_fdk_filter(
            p.data_ptr(), A, U, V, float(pixel_size), sod.data_ptr(), sid.data_ptr(), float(alpha),
            out.data_ptr(), _p(ws), 0 if ws is None else ws.numel(), _stream(dev)))
    return out


def fdk_filter_backward(grad_filtered, projections, filtered, pixel_size, sod, sid, alpha,
                        need_projections=True, need_distances=True):
    """Gradients of ``fdk_filter`` (dgc_fdk_filter_backward): ``(grad_projections,
    grad_sod, grad_sid)``, each None when not asked for."""
    g = grad_filtered.contiguous()
    A, U, V = g.shape
    dev = g.device
    gp = torch.empty_like(g) if need_projections else None
    gsod = torch.empty((A,), dtype=torch.float32, device=dev) if need_distances else None
    gsid = torch.empty((A,), dtype=torch.float32, device=dev) if need_distances else None
    p = projections.contiguous() if need_distances else None
    y = filtered.contiguous() if need_distances else None
    lib = _native.lib()
    with torch.cuda.device(dev):
        ws = _workspace(lib.dgc_fdk_filter_backward_workspace_bytes(A, U, V), dev)
        _native.check(lib.dgc_fdk_filter_backward(
            g.data_ptr(), _p(p), _p(y), A, U, V, float(pixel_size), sod.data_ptr(),
            sid.data_ptr(), float(alpha), _p(gp), _p(gsod), _p(gsid), _p(ws),
            0 if ws is None else ws.numel(), _stream(dev)))
    return gp, gsod, gsid


def _frame(frame):
    """A preweight frame (dist, u, v) as contiguous tensors (None entries kept)."""
    frame = (None, None, None) if frame is None else tuple(frame)
    _require(len(frame) == 3, "a preweight frame is (dist, u, v)")
    return [None if t is None else t.contiguous() for t in frame]


def fdk_filter_framed(projections, pixel_size, sod, sid, alpha, frame):
    """``fdk_filter`` with the cosine preweight in a per-view frame
    (dgc_fdk_filter_ex): ``frame = (dist, u, v)``, each a CUDA float32 [A]
    tensor or None (sid, (U-1)/2, (V-1)/2)."""
    A, U, V = projections.shape
    p = projections.contiguous()
    dev = p.device
    frame = _frame(frame)
    ptrs = [_p(t) for t in frame]
    out = torch.empty_like(p)
    lib = _native.lib()
    with torch.cuda.device(dev):
        ws = _workspace(lib.dgc_fdk_filter_workspace_bytes(A, U, V), dev)
        _native.check(lib.dgc_fdk_filter_ex(
            p.data_ptr(), A, U, V, float(pixel_size), sod.data_ptr(), sid.data_ptr(), *ptrs,
            float(alpha), out.data_ptr(), _p(ws), 0 if ws is None else ws.numel(),
            _stream(dev)))
    return out


def fdk_filter_backward_framed(grad_filtered, projections, filtered, pixel_size, sod, sid, alpha,
                               frame, need_projections, need_sod, need_sid, need_frame):
    """Gradients of ``fdk_filter_framed`` (dgc_fdk_filter_backward_ex):
    ``(grad_projections, grad_sod, grad_sid, grad_dist, grad_u, grad_v)``,
    each None when not asked for (``need_frame`` three flags)."""
    g = grad_filtered.contiguous()
    A, U, V = g.shape
    dev = g.device
    frame = _frame(frame)
    ptrs = [_p(t) for t in frame]

    def vec(need):
        return torch.empty((A,), dtype=torch.float32, device=dev) if need else None

    gp = torch.empty_like(g) if need_projections else None
    gsod, gsid = vec(need_sod), vec(need_sid)
    gframe = [vec(n and t is not None) for n, t in zip(need_frame, frame)]
    dist = need_sod or need_sid or any(t is not None for t in gframe)
    p = projections.contiguous() if dist else None
    y = filtered.contiguous() if dist else None
    lib = _native.lib()
    with torch.cuda.device(dev):
        ws = _workspace(lib.dgc_fdk_filter_backward_workspace_bytes(A, U, V), dev)
        _native.check(lib.dgc_fdk_filter_backward_ex(
            g.data_ptr(), _p(p), _p(y), A, U, V, float(pixel_size), sod.data_ptr(),
            sid.data_ptr(), *ptrs, float(alpha), _p(gp), _p(gsod), _p(gsid),
            *[_p(t) for t in gframe], _p(ws), 0 if ws is None else ws.numel(), _stream(dev)))
    return (gp, gsod, gsid, *gframe)


def reconstruct_fdk_ex(projections, geometry, pixel_size, volume_shape, voxel_size, volume_offset,
                       alpha, frame, uweights, angle_scale, clamp=True):
    """The general reconstruction (dgc_reconstruct_fdk_ex): preweight frame
    ``frame`` (or None), per-(view, column) weights ``uweights`` (or None),
    angular factor ``angle_scale``, optional clamp."""
    p = projections.contiguous()
    geom = [t.contiguous() for t in geometry]
    w = None if uweights is None else uweights.contiguous()
    frame = _frame(frame)
    ptrs = [_p(t) for t in frame]
    A, U, V = p.shape
    D, H, W = volume_shape
    dev = p.device
    vol = torch.empty((D, H, W), dtype=torch.float32, device=dev)
    lib = _native.lib()
    with torch.cuda.device(dev):
        ws = _workspace(lib.dgc_reconstruct_fdk_workspace_bytes(A, U, V, D, H, W), dev)
        _native.check(lib.dgc_reconstruct_fdk_ex(
            p.data_ptr(), A, U, V, *[g.data_ptr() for g in geom], float(pixel_size), D, H, W,
            float(voxel_size), *map(float, volume_offset), float(alpha), *ptrs, _p(w),
            float(angle_scale), 1 if clamp else 0, vol.data_ptr(), _p(ws),
            0 if ws is None else ws.numel(), _stream(dev)))
    return vol


def reconstruct_fdk(projections, geometry, pixel_size, volume_shape, voxel_size, volume_offset,
                    alpha):
    """Filter + backproject all views, * pi/A, clamp at 0, in two kernels."""
    p = projections.contiguous()
    geom = [t.contiguous() for t in geometry]
    A, U, V = p.shape
    D, H, W = volume_shape
    dev = p.device
    vol = torch.empty((D, H, W), dtype=torch.float32, device=dev)
    lib = _native.lib()
    with torch.cuda.device(dev):
        ws = _workspace(lib.dgc_reconstruct_fdk_workspace_bytes(A, U, V, D, H, W), dev)
        _native.check(lib.dgc_reconstruct_fdk(
            p.data_ptr(), A, U, V, *[g.data_ptr() for g in geom], float(pixel_size), D, H, W,
            float(voxel_size), *map(float, volume_offset), float(alpha), vol.data_ptr(), _p(ws),
            0 if ws is None else ws.numel(), _stream(dev)))
    return vol


def parker_weights(angles, sid, U, pixel_size, frame_dist=None, frame_u=None):
    """float32 [A,U] Parker short-scan weights of the scan ``angles``
    (dgc_parker_weights; dgc_parker_weights_ex with fan angles taken in a
    preweight frame when ``frame_dist`` / ``frame_u`` are given)."""
    a = angles.contiguous()
    d = sid.contiguous()
    A = a.numel()
    out = torch.empty((A, int(U)), dtype=torch.float32, device=a.device)
    lib = _native.lib()
    with torch.cuda.device(a.device):
        if frame_dist is None and frame_u is None:
            _native.check(lib.dgc_parker_weights(a.data_ptr(), d.data_ptr(), A, int(U),
                                                 float(pixel_size), out.data_ptr(),
                                                 _stream(a.device)))
        else:
            fd = None if frame_dist is None else frame_dist.contiguous()
            fu = None if frame_u is None else frame_u.contiguous()
            _native.check(lib.dgc_parker_weights_ex(a.data_ptr(), d.data_ptr(), _p(fd), _p(fu),
                                                    A, int(U), float(pixel_size),
                                                    out.data_ptr(), _stream(a.device)))
    return out


def reconstruct_fdk_weighted(projections, geometry, pixel_size, volume_shape, voxel_size,
                             volume_offset, alpha, uweights, angle_scale):
    """reconstruct_fdk with per-(view, column) weights and angular factor
    ``angle_scale`` in place of pi/A (short scans)."""
    p = projections.contiguous()
    geom = [t.contiguous() for t in geometry]
    w = None if uweights is None else uweights.contiguous()
    A, U, V = p.shape
    D, H, W = volume_shape
    dev = p.device
    vol = torch.empty((D, H, W), dtype=torch.float32, device=dev)
    lib = _native.lib()
    with torch.cuda.device(dev):
        ws = _workspace(lib.dgc_reconstruct_fdk_workspace_bytes(A, U, V, D, H, W), dev)
        _native.check(lib.dgc_reconstruct_fdk_weighted(
            p.data_ptr(), A, U, V, *[g.data_ptr() for g in geom], float(pixel_size), D, H, W,
            float(voxel_size), *map(float, volume_offset), float(alpha), _p(w),
            float(angle_scale), vol.data_ptr(), _p(ws), 0 if ws is None else ws.numel(),
            _stream(dev)))
    return vol


def reconstruct_fdk_partial(projections, geometry, pixel_size, volume_shape, voxel_size,
                            volume_offset, alpha, uweights, angle_scale):
    """This rank's unclamped share of a view-sharded reconstruction
    (dgc_reconstruct_fdk_partial): filter + backproject its views, times
    ``angle_scale``."""
    p = projections.contiguous()
    geom = [t.contiguous() for t in geometry]
    w = None if uweights is None else uweights.contiguous()
    A, U, V = p.shape
    D, H, W = volume_shape
    dev = p.device
    vol = torch.empty((D, H, W), dtype=torch.float32, device=dev)
    lib = _native.lib()
    with torch.cuda.device(dev):
        ws = _workspace(lib.dgc_reconstruct_fdk_workspace_bytes(A, U, V, D, H, W), dev)
        _native.check(lib.dgc_reconstruct_fdk_partial(
            p.data_ptr(), A, U, V, *[g.data_ptr() for g in geom], float(pixel_size), D, H, W,
            float(voxel_size), *map(float, volume_offset), float(alpha), _p(w),
            float(angle_scale), vol.data_ptr(), _p(ws), 0 if ws is None else ws.numel(),
            _stream(dev)))
    return vol


def clamp_volume(volume):
    """In-place clamp at zero (dgc_clamp_volume) of a contiguous float32 CUDA volume."""
    _require(volume.is_cuda and volume.dtype == torch.float32 and volume.is_contiguous(),
             "volume must be a contiguous float32 CUDA tensor")
    with torch.cuda.device(volume.device):
        _native.check(_native.lib().dgc_clamp_volume(volume.data_ptr(), volume.numel(),
                                                     _stream(volume.device)))
    return volume


def fdk_filter_taps(U: int, pixel_size: float, alpha: float):
    """Host-only filter taps h[0..U-1] (FP64), for inspection and tests."""
    import ctypes

    buf = (ctypes.c_double * int(U))()
    _native.check(_native.lib().dgc_fdk_filter_taps(int(U), float(pixel_size), float(alpha), buf))
    return list(buf)


def project_sample_counts(volume_shape, geometry, pixel_size, U, V, step_size, voxel_size,
                          offset=(0.0, 0.0, 0.0)):
    """int64 [A,U,V] number of trilinear samples per ray (FP32 stepping rule)."""
    geom = [t.contiguous() for t in geometry]
    A = geom[0].numel()
    D, H, W = volume_shape
    dev = geom[0].device
    out = torch.empty((A, int(U), int(V)), dtype=torch.int64, device=dev)
    with torch.cuda.device(dev):
        _native.check(_native.lib().dgc_project_sample_counts(
            D, H, W, *[g.data_ptr() for g in geom], A, float(pixel_size), int(U), int(V),
            float(step_size), float(voxel_size), *map(float, offset), out.data_ptr(), _stream(dev)))
    return out
