"""ctypes front end of the FP64 CPU oracle (``oracle/dgc_oracle.c``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, by ``__graft_entry__.smoke()``
and by the CPU-baseline leg of ``bench.py`` as the checker.  The product package
never imports it.

Every function takes numpy arrays (any float dtype; converted to contiguous
float64) and returns float64 results.  Geometry is given as the reference's
eight per-view arrays ``(angles, sid, sod, det_u0, det_v0, src_x, src_y, src_z)``.
The algorithms restate the reference project's kernels and CPU checks; the C
file cites the reference lines each function follows.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_lib" / "libdgc_oracle.so"

_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)
_c_int = ctypes.c_int
_c_long = ctypes.c_long
_c_d = ctypes.c_double

_lib = None


def build(force: bool = False) -> Path:
    """Compile the oracle with its Makefile (gcc); returns the library path."""
    src = HERE / "dgc_oracle.c"
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def _load():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        lib = ctypes.CDLL(str(LIB_PATH))
        fp_args = [_c_int, _c_int, _c_int, _dp, _c_int, _c_int, _c_int, _c_d, _c_d, _c_d,
                   _c_d, _c_d, _c_d, _c_int]
        lib.oracle_project.argtypes = [_dp] + fp_args + [_dp]
        lib.oracle_project_rays.argtypes = [_dp] + fp_args + [_i64p, _c_long, _dp]
        lib.oracle_sample_counts.argtypes = fp_args + [_i64p]
        lib.oracle_ray_traces.argtypes = fp_args + [_c_d, _i64p]
        lib.oracle_project_backward.argtypes = [_dp, _dp] + fp_args + [_dp, _dp]
        bp_args = [_c_int, _c_int, _c_int, _dp, _c_d, _c_int, _c_int, _c_int, _c_d, _c_d,
                   _c_d, _c_d]
        lib.oracle_backproject.argtypes = [_dp] + bp_args + [_dp]
        lib.oracle_backproject_backward.argtypes = [_dp, _dp] + bp_args + [_dp, _dp]
        lib.oracle_fdk_taps.argtypes = [_c_int, _c_d, _c_d, _dp]
        lib.oracle_fdk_filter.argtypes = [_dp, _c_int, _c_int, _c_int, _c_d, _dp, _dp, _c_d, _dp]
        lib.oracle_fdk_filter_frame.argtypes = [_dp, _c_int, _c_int, _c_int, _c_d, _dp, _dp, _dp,
                                                _dp, _dp, _c_d, _dp]
        lib.oracle_num_threads.restype = _c_int
        lib.oracle_set_num_threads.argtypes = [_c_int]
        env = os.environ.get("DGC_ORACLE_THREADS")
        lib.oracle_set_num_threads(int(env) if env else usable_cpus())
        _lib = lib
    return _lib


def _f64(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


def _ptr(a):
    return a.ctypes.data_as(_dp)


def _geom(geometry, A=None):
    g = np.stack([_f64(np.asarray(x).reshape(-1)) for x in geometry])
    if g.shape[0] != 8:
        raise ValueError("geometry must hold 8 per-view arrays")
    if A is not None and g.shape[1] != A:
        raise ValueError("geometry arrays must have A entries")
    return np.ascontiguousarray(g)


def num_threads() -> int:
    return _load().oracle_num_threads()


def set_num_threads(n: int) -> None:
    _load().oracle_set_num_threads(int(n))


def project(volume, geometry, pixel_size, U, V, step_size, voxel_size,
            offset=(0.0, 0.0, 0.0), mode=0):
    """Forward projection [A,U,V]; ``mode`` 0 = reference CPU rule, 1 = FP32 kernel sample set."""
    vol = _f64(volume)
    D, H, W = vol.shape
    g = _geom(geometry)
    A = g.shape[1]
    out = np.empty((A, U, V), np.float64)
    _load().oracle_project(_ptr(vol), D, H, W, _ptr(g), A, U, V, pixel_size, step_size,
                           voxel_size, *map(float, offset), int(mode), _ptr(out))
    return out


def project_rays(volume, geometry, pixel_size, U, V, step_size, voxel_size, rays,
                 offset=(0.0, 0.0, 0.0), mode=0):
    """Forward projection of selected rays (flat indices ``(a*U+u)*V+v``)."""
    vol = _f64(volume)
    D, H, W = vol.shape
    g = _geom(geometry)
    A = g.shape[1]
    r = np.ascontiguousarray(np.asarray(rays, dtype=np.int64))
    out = np.empty(r.shape[0], np.float64)
    _load().oracle_project_rays(_ptr(vol), D, H, W, _ptr(g), A, U, V, pixel_size, step_size,
                                voxel_size, *map(float, offset), int(mode),
                                r.ctypes.data_as(_i64p), r.shape[0], _ptr(out))
    return out


def sample_counts(volume_shape, geometry, pixel_size, U, V, step_size, voxel_size,
                  offset=(0.0, 0.0, 0.0), mode=1):
    D, H, W = volume_shape
    g = _geom(geometry)
    A = g.shape[1]
    out = np.empty((A, U, V), np.int64)
    _load().oracle_sample_counts(D, H, W, _ptr(g), A, U, V, pixel_size, step_size, voxel_size,
                                 *map(float, offset), int(mode), out.ctypes.data_as(_i64p))
    return out


def ray_traces(volume_shape, geometry, pixel_size, U, V, step_size, voxel_size,
               offset=(0.0, 0.0, 0.0), mode=1, margin=1e-4):
    """uint64 [A,U,V] hash of (entry face, sample count, cells); 0 = near a cell boundary."""
    D, H, W = volume_shape
    g = _geom(geometry)
    A = g.shape[1]
    out = np.empty((A, U, V), np.int64)
    _load().oracle_ray_traces(D, H, W, _ptr(g), A, U, V, pixel_size, step_size, voxel_size,
                              *map(float, offset), int(mode), float(margin),
                              out.ctypes.data_as(_i64p))
    return out.view(np.uint64)


def project_backward(grad_projection, volume, geometry, pixel_size, step_size, voxel_size,
                     offset=(0.0, 0.0, 0.0), mode=0, compute_grad_volume=True):
    """Analytic gradients: (grad_volume or None, [8, A] geometry gradients)."""
    gp = _f64(grad_projection)
    vol = _f64(volume)
    D, H, W = vol.shape
    A, U, V = gp.shape
    g = _geom(geometry, A)
    gv = np.empty_like(vol) if compute_grad_volume else None
    gg = np.empty((8, A), np.float64)
    _load().oracle_project_backward(
        _ptr(gp), _ptr(vol), D, H, W, _ptr(g), A, U, V, pixel_size, step_size, voxel_size,
        *map(float, offset), int(mode), _ptr(gv) if gv is not None else None, _ptr(gg))
    return gv, gg


def backproject(projections, geometry, pixel_size, volume_shape, voxel_size,
                offset=(0.0, 0.0, 0.0)):
    p = _f64(projections)
    A, U, V = p.shape
    g = _geom(geometry, A)
    D, H, W = volume_shape
    out = np.empty((D, H, W), np.float64)
    _load().oracle_backproject(_ptr(p), A, U, V, _ptr(g), pixel_size, D, H, W, voxel_size,
                               *map(float, offset), _ptr(out))
    return out


def backproject_backward(grad_volume, projections, geometry, pixel_size, voxel_size,
                         offset=(0.0, 0.0, 0.0)):
    """Analytic gradients: (grad_projections [A,U,V], [8, A] geometry gradients)."""
    gv = _f64(grad_volume)
    p = _f64(projections)
    A, U, V = p.shape
    D, H, W = gv.shape
    g = _geom(geometry, A)
    gp = np.empty_like(p)
    gg = np.empty((8, A), np.float64)
    _load().oracle_backproject_backward(_ptr(gv), _ptr(p), A, U, V, _ptr(g), pixel_size, D, H,
                                        W, voxel_size, *map(float, offset), _ptr(gp), _ptr(gg))
    return gp, gg


def fdk_taps(U, pixel_size, alpha=0.8):
    h = np.empty(U, np.float64)
    _load().oracle_fdk_taps(int(U), float(pixel_size), float(alpha), _ptr(h))
    return h


def fdk_filter(projections, pixel_size, sod, sid, alpha=0.8, frame=None):
    """filtering.py:54-104 in FP64; ``frame = (dist, u, v)`` (each None, a
    scalar or [A]) takes the cosine preweight in that frame instead of the
    centred one (no counterpart in the reference)."""
    p = _f64(projections)
    A, U, V = p.shape

    def per_view(x):
        return _f64(np.broadcast_to(np.asarray(x, np.float64).reshape(-1), (A,)))

    sod, sid = per_view(sod), per_view(sid)
    out = np.empty_like(p)
    if frame is None:
        _load().oracle_fdk_filter(_ptr(p), A, U, V, float(pixel_size), _ptr(sod), _ptr(sid),
                                  float(alpha), _ptr(out))
        return out
    fr = [None if x is None else per_view(x) for x in frame]
    ptrs = [_dp() if x is None else _ptr(x) for x in fr]
    _load().oracle_fdk_filter_frame(_ptr(p), A, U, V, float(pixel_size), _ptr(sod), _ptr(sid),
                                    *ptrs, float(alpha), _ptr(out))
    return out


def fdk_filter_backward(grad_filtered, projections, pixel_size, sod, sid, alpha=0.8,
                        frame=None):
    """FP64 gradients of ``fdk_filter`` for the upstream gradient g, restated
    analytically: with y = c H(w P), c = px sid/sod, w = D/r, r^2 = D^2 +
    u_c^2 + v_c^2 (D = frame dist or sid, u_c, v_c the pixel's offsets from
    the frame centre in length units) and z = H g (H symmetric Toeplitz):
    grad P = c w z; grad sod = -sum(g y)/sod; grad sid = sum(g y)/sid, plus
    c sum(z P (u_c^2+v_c^2)/r^3) when D is sid; grad D = c sum(z P
    (u_c^2+v_c^2)/r^3); grad u = c D px sum(z P u_c/r^3), grad v likewise.
    Returns a dict of float64 arrays (``P``, ``sod``, ``sid`` and, for the
    frame entries given, ``dist``, ``u``, ``v``)."""
    g = _f64(grad_filtered)
    p = _f64(projections)
    A, U, V = p.shape

    def per_view(x):
        return np.broadcast_to(np.asarray(x, np.float64).reshape(-1), (A,)).copy()

    sod, sid = per_view(sod), per_view(sid)
    fr = (None, None, None) if frame is None else tuple(frame)
    dist = sid if fr[0] is None else per_view(fr[0])
    cu = np.full(A, (U - 1) / 2.0) if fr[1] is None else per_view(fr[1])
    cv = np.full(A, (V - 1) / 2.0) if fr[2] is None else per_view(fr[2])
    h = fdk_taps(U, pixel_size, alpha)
    idx = np.arange(U)
    H = h[np.abs(idx[:, None] - idx[None, :])]
    y = fdk_filter(p, pixel_size, sod, sid, alpha, frame)
    out = {k: np.empty(A) for k in ("sod", "sid", "dist", "u", "v")}
    out["P"] = np.empty_like(p)
    for a in range(A):
        uc = (idx - cu[a]) * pixel_size
        vc = (np.arange(V) - cv[a]) * pixel_size
        r2 = uc[:, None] ** 2 + vc[None, :] ** 2
        r = np.sqrt(dist[a] ** 2 + r2)
        w = dist[a] / r
        c = pixel_size * sid[a] / sod[a]
        z = H @ g[a]
        out["P"][a] = c * w * z
        gy = float((g[a] * y[a]).sum())
        zp = z * p[a]
        zpw = float((zp * r2 / r ** 3).sum())
        out["sod"][a] = -gy / sod[a]
        out["sid"][a] = gy / sid[a] + (0.0 if fr[0] is not None else c * zpw)
        out["dist"][a] = c * zpw
        out["u"][a] = c * dist[a] * pixel_size * float((zp * uc[:, None] / r ** 3).sum())
        out["v"][a] = c * dist[a] * pixel_size * float((zp * vc[None, :] / r ** 3).sum())
    for k, x in zip(("dist", "u", "v"), fr):
        if x is None:
            del out[k]
    return out


def preweight_frame(geometry, pixel_size):
    """FP64 (dist, u, v) per view: the source's distance to the detector plane
    and the pixel indices of the foot of its perpendicular, from the
    projector's source and detector points (fp.cu:115-170 as restated in
    ``dgc_oracle.c``): source O = (-sod sin b + sx, sod cos b + sy, sz),
    detector point T(u, v) = ((u-u0) px cos b - (sod-sid) sin b,
    (u-u0) px sin b + (sod-sid) cos b, (v-v0) px)."""
    g = _geom(geometry)
    b, sid, sod, u0, v0, sx, sy, sz = g
    ds_u = sx * np.cos(b) + sy * np.sin(b)
    ds_n = -sx * np.sin(b) + sy * np.cos(b)
    return sid + ds_n, u0 + ds_u / pixel_size, v0 + sz / pixel_size


def parker_weights(angles, sid, U, pixel_size, frame_dist=None, frame_u=None):
    """FP64 [A,U] short-scan weights (Parker, Med. Phys. 9(2), 1982), as
    dgc_parker_weights defines them: beta from angles[0] in the scan's
    direction, Gamma = (range - pi) / 2, gamma = atan(u_c / sid) with the
    centred u_c of filtering.py's cosine preweight, gamma's sign following the
    scan direction.  ``frame_dist`` / ``frame_u`` replace sid and the centre
    (U-1)/2 in gamma (the offset-aware preweight frame)."""
    a = np.asarray(angles, np.float64)
    d = np.broadcast_to(np.asarray(sid if frame_dist is None else frame_dist, np.float64),
                        a.shape)
    centre = np.broadcast_to(np.asarray(0.5 * (U - 1) if frame_u is None else frame_u,
                                        np.float64), a.shape)
    direction = 1.0 if a[-1] >= a[0] else -1.0
    beta = (direction * (a - a[0]))[:, None]
    gam_max = 0.5 * (direction * (a[-1] - a[0]) - np.pi)
    uc = (np.arange(U)[None, :] - centre[:, None]) * pixel_size
    gam = direction * np.arctan(uc / d[:, None])
    w = np.zeros((a.size, U))
    with np.errstate(divide="ignore", invalid="ignore"):
        rise = np.sin(0.25 * np.pi * beta / (gam_max - gam)) ** 2
        fall = np.sin(0.25 * np.pi * (np.pi + 2 * gam_max - beta) / (gam_max + gam)) ** 2
    r1 = (beta >= 0) & (beta < 2 * (gam_max - gam))
    r2 = ~r1 & (beta >= 0) & (beta <= np.pi - 2 * gam)
    r3 = (beta > np.pi - 2 * gam) & (beta <= np.pi + 2 * gam_max)
    w = np.where(r1, rise, w)
    w = np.where(r2, 1.0, w)
    w = np.where(r3 & ~r1 & ~r2, fall, w)
    return w


def reconstruct_fdk(projections, geometry, pixel_size, volume_shape, voxel_size,
                    offset=(0.0, 0.0, 0.0), alpha=0.8, offset_preweight=False):
    """filtering.py:107-198 in FP64: filter, backproject, * pi/A, clamp >= 0
    (``offset_preweight``: the cosine preweight in ``preweight_frame``)."""
    g = _geom(geometry)
    frame = preweight_frame(g, pixel_size) if offset_preweight else None
    filtered = fdk_filter(projections, pixel_size, g[2], g[1], alpha, frame)
    vol = backproject(filtered, g, pixel_size, volume_shape, voxel_size, offset)
    return np.maximum(vol * (np.pi / g.shape[1]), 0.0)


__all__ = [
    "build", "num_threads", "set_num_threads", "project", "project_rays", "sample_counts",
    "ray_traces", "project_backward", "backproject", "backproject_backward", "fdk_taps", "fdk_filter",
    "reconstruct_fdk", "parker_weights", "preweight_frame", "fdk_filter_backward", "usable_cpus",
]


def usable_cpus() -> int:
    """CPUs this process may use: its affinity set, capped by a cgroup-v2 CPU
    quota (cpu.max) when one is set -- the count of online processors can be
    far larger inside a container."""
    try:
        n = len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        n = os.cpu_count() or 1
    try:
        quota, period = open("/sys/fs/cgroup/cpu.max").read().split()[:2]
        if quota != "max":
            n = min(n, max(1, -(-int(quota) // int(period))))
    except (OSError, ValueError):
        pass
    return max(1, n)

