"""Per-view geometry calibration by gradient descent through ``project``.

The reference project names a geometry-calibration pipeline but does not ship
it (its README and docs/SOURCE.md); what it ships is the differentiable
projector whose nine gradients make calibration possible.  This module builds
the plain calibration loop on top of this library's operators:

* ``perturb_geometry``: per-view perturbations of a nominal circular scan
  (angle, source offsets, detector centre, sid/sod scale) drawn from a seed;
* ``simulate_measurement``: line integrals through the true geometry, Poisson
  counts at ``I0`` photons, ``-log`` back to line integrals, and the mask of
  rays with usable counts (photon-starved rays carry no geometry information:
  their ``-log`` saturates near ``log(I0)``);
* ``reprojection_error``: RMS detector distance (pixels) between where a fixed
  lattice of 3-D points lands under two geometries, with the backprojector's
  voxel-to-detector mapping (src_cbct_backprojector_cuda.cu:48-72 of the
  reference) -- the success metric, insensitive to the near-degenerate
  directions of the per-view parameters (angle vs det_u0 vs src_x, sid vs sod);
* ``calibrate``: Adam on per-view offsets ``delta`` of the eight geometry
  tensors, minimising ``MSE(project(volume, nominal + delta), measured)``,
  optionally from a warm start that is rejected if it raises that loss.  By
  default each step is one fused kernel pass (``dgc_project_mse_grad``:
  projection, masked squared error and the eight geometry gradients from one
  ray march) instead of ``project`` + autograd backward (two marches).

All arithmetic on the device; the projector and its geometry gradients run in
``libdgc.so``.
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import torch

from . import _ops
from .source_only_forward_projector import project

GEOMETRY_NAMES = ("angles", "sid", "sod", "det_u0", "det_v0", "src_x", "src_y", "src_z")

# Adam step sizes per parameter family (radians, length units, pixels): the
# per-iteration move Adam makes is about this size.  Chosen on held-out
# stacks of the 128^3 / 180 view / 256^2 acquisition (0.1 px RMS reprojection
# error in 46-52 iterations) and confirmed on 256^3 / 360 views / 384^2 (71).
DEFAULT_LR = {"angles": 3e-3, "sid": 3.0, "sod": 3.0, "det_u0": 0.3, "det_v0": 0.3,
              "src_x": 0.3, "src_y": 0.3, "src_z": 0.3}


@dataclass
class ScanSetup:
    """Scalar acquisition settings shared by every view."""

    U: int
    V: int
    pixel_size: float = 1.0
    step_size: float = 0.5
    voxel_size: float = 1.0
    volume_offset: tuple = (0.0, 0.0, 0.0)


def perturb_geometry(nominal, seed, angle_deg=0.3, src_mm=1.0, det_px=2.0, dist_rel=0.005):
    """True per-view geometry: nominal + N(0, sigma) per view and family (config-3 model)."""
    g = torch.Generator(device="cpu").manual_seed(int(seed))
    A = nominal[0].numel()

    def n(scale):
        return (torch.randn(A, generator=g, dtype=torch.float64) * scale).to(
            nominal[0].device, torch.float32)

    angles, sid, sod, u0, v0, sx, sy, sz = nominal
    return [angles + n(math.radians(angle_deg)),
            sid * (1.0 + n(dist_rel)),
            sod * (1.0 + n(dist_rel)),
            u0 + n(det_px), v0 + n(det_px),
            sx + n(src_mm), sy + n(src_mm), sz + n(src_mm)]


@torch.no_grad()
def simulate_measurement(volume, geometry, scan: ScanSetup, I0=1e5, seed=0, min_counts=50):
    """Measured line integrals and the mask of usable rays.

    Returns ``(-log(Poisson(I0 * exp(-p)) / I0), mask)`` with p the projections
    under ``geometry`` and ``mask`` = 1 where the counts reach ``min_counts``
    (all ones when ``I0`` is None: noiseless line integrals).
    """
    p = project(volume, *geometry, scan.pixel_size, scan.U, scan.V, step_size=scan.step_size,
                voxel_size=scan.voxel_size, off_x=scan.volume_offset[0],
                off_y=scan.volume_offset[1], off_z=scan.volume_offset[2])
    if I0 is None:
        return p, torch.ones_like(p)
    gen = torch.Generator(device=p.device).manual_seed(int(seed))
    counts = torch.poisson(I0 * torch.exp(-p.double()), generator=gen)
    mask = (counts >= min_counts).float()
    return (-torch.log(counts.clamp_min(1.0) / I0)).float(), mask


def lattice_points(volume_shape, voxel_size=1.0, offset=(0.0, 0.0, 0.0), n=8, extent=0.7,
                   device="cuda"):
    """(x, y, z) of an n^3 lattice spanning ``extent`` of the volume, world units."""
    D, H, W = volume_shape
    axes = []
    for size, off in ((W, offset[0]), (H, offset[1]), (D, offset[2])):
        half = 0.5 * extent * size * voxel_size
        axes.append(torch.linspace(-half, half, n, device=device, dtype=torch.float64) + off)
    z, y, x = torch.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    return torch.stack([x.reshape(-1), y.reshape(-1), z.reshape(-1)], 1)


def detector_coordinates(points, geometry, pixel_size):
    """[A, P, 2] detector indices (u_idx, v_idx) of world points, FP64.

    The voxel-to-detector mapping of the backprojector (bp.cu:48-72).
    """
    angles, sid, sod, u0, v0, sx, sy, sz = (t.double()[:, None] for t in geometry)
    x, y, z = (points[:, k][None, :] for k in range(3))
    c, s = torch.cos(angles), torch.sin(angles)
    px, py = x * c + y * s, -x * s + y * c
    ds_u, ds_n = sx * c + sy * s, -sx * s + sy * c
    t = (sid + ds_n) / (sod + ds_n - py)
    u = (ds_u + t * (px - ds_u)) / pixel_size + u0
    v = (sz + t * (z - sz)) / pixel_size + v0
    return torch.stack([u, v], -1)


def reprojection_error(geometry_a, geometry_b, points, pixel_size):
    """RMS over views and points of the detector distance [pixels]."""
    da = detector_coordinates(points, geometry_a, pixel_size)
    db = detector_coordinates(points, geometry_b, pixel_size)
    return float((da - db).square().sum(-1).mean().sqrt())


def angle_error_deg(geometry_a, geometry_b):
    """RMS angle difference [degrees]."""
    d = (geometry_a[0].double() - geometry_b[0].double())
    return float(torch.rad2deg(d).square().mean().sqrt())


def _metric_terms(geometry_a, geometry_b, points, pixel_size):
    """FP64 [4]: sum and count of the squared detector distances and of the
    squared angle differences (the RMS metrics before the mean), so that
    ranks holding different views can add them up."""
    da = detector_coordinates(points, geometry_a, pixel_size)
    db = detector_coordinates(points, geometry_b, pixel_size)
    sq = (da - db).square().sum(-1)
    dang = torch.rad2deg(geometry_a[0].double() - geometry_b[0].double())
    return torch.stack([sq.sum(), torch.tensor(float(sq.numel()), dtype=torch.float64,
                                                 device=sq.device),
                        dang.square().sum(), torch.tensor(float(dang.numel()),
                                                          dtype=torch.float64, device=sq.device)])


@dataclass
class CalibrationResult:
    delta: list
    geometry: list
    history: list = field(default_factory=list)
    time_to_target_s: float | None = None
    iterations_to_target: int | None = None
    warm_start_accepted: bool | None = None
    final_loss: float = float("nan")


def _loss_terms(volume, geometry, measured, scan, mask=None):
    """(sum of the squared mismatch over the usable rays, their count)."""
    p = project(volume, *geometry, scan.pixel_size, scan.U, scan.V, step_size=scan.step_size,
                voxel_size=scan.voxel_size, off_x=scan.volume_offset[0],
                off_y=scan.volume_offset[1], off_z=scan.volume_offset[2])
    r = (p - measured).square()
    if mask is None:
        return r.sum(), torch.tensor(float(r.numel()), device=r.device)
    return (r * mask).sum(), mask.sum()


def _loss(volume, geometry, measured, scan, mask=None):
    """Mean squared projection mismatch over the usable rays."""
    p = project(volume, *geometry, scan.pixel_size, scan.U, scan.V, step_size=scan.step_size,
                voxel_size=scan.voxel_size, off_x=scan.volume_offset[0],
                off_y=scan.volume_offset[1], off_z=scan.volume_offset[2])
    r = (p - measured).square()
    if mask is None:
        return r.mean()
    return (r * mask).sum() / mask.sum().clamp_min(1.0)


class _FusedMSE(torch.autograd.Function):
    """Masked MSE of the projection as a function of the eight geometry
    tensors; value and gradients from one fused kernel pass."""

    @staticmethod
    def forward(ctx, volume, measured, mask, scale, scan, *geometry):
        loss, grads, _ = _ops.fp_mse_grad(volume, geometry, scan.pixel_size, scan.U, scan.V,
                                          scan.step_size, scan.voxel_size, measured, mask, scale,
                                          scan.volume_offset)
        ctx.save_for_backward(*grads)
        return loss.float()

    @staticmethod
    def backward(ctx, grad_loss):
        return (None, None, None, None, None, *[g * grad_loss for g in ctx.saved_tensors])


def _fused_loss(volume, geometry, measured, scan, mask=None, denom=None):
    if denom is None:
        denom = float(measured.numel() if mask is None else mask.sum().clamp_min(1.0))
    return _FusedMSE.apply(volume, measured, mask, 1.0 / denom, scan, *geometry)


def calibrate(volume, measured, nominal, scan: ScanSetup, iterations=200, lr=None,
              warm_start=None, true_geometry=None, points=None, target_px=0.1,
              target_angle_deg=None, stop_at_target=False, log_every=0, mask=None,
              final_lr_fraction=1.0, lr_gamma=1.0, decay_start=0, fused=True,
              warmup_iterations=0, betas=(0.9, 0.99), reduce=None):
    """Adam on per-view geometry offsets; returns a ``CalibrationResult``.

    The loss is the mean squared mismatch between ``project(volume, nominal +
    delta)`` and ``measured`` over the rays where ``mask`` is 1 (all rays when
    ``mask`` is None).  Step sizes follow a cosine decay to
    ``final_lr_fraction`` of their start over ``iterations`` (1.0: constant),
    times ``lr_gamma ** max(0, it - decay_start)``, ramped up linearly over
    the first ``warmup_iterations`` (Adam's first steps are ``lr``-sized
    whatever the gradient, which throws a good start away).  ``fused`` selects the
    one-pass loss-and-gradient kernel (default) or ``project`` + autograd.

    ``warm_start`` (8 tensors [A], e.g. a network's prediction) is used as the
    initial delta only if it does not raise the projection loss relative to
    the nominal start; otherwise calibration starts from nominal.  When
    ``true_geometry`` is given, the reprojection error is tracked every
    iteration and the wall time to ``target_px`` (and ``target_angle_deg``) is
    recorded, counted from the call (network inference happens before it and is
    the caller's to add).

    ``reduce`` (view sharding, ``sharded.calibrate_sharded``): each caller
    holds only its own views, and ``reduce`` sums an FP64 tensor over all of
    them; the loss normalisation, the warm-start judge, the recorded loss and
    the metrics are then those of the whole scan.  The views' offsets are
    independent, so every rank's steps equal those of one calibration over all
    views.
    """
    t0 = time.perf_counter()
    lr = dict(DEFAULT_LR, **(lr or {}))
    volume = volume.detach()
    measured = measured.detach()
    nominal = [g.detach() for g in nominal]
    delta = [torch.zeros_like(g) for g in nominal]
    accepted = None

    def loss_of(geometry):
        if reduce is None:
            return float(_loss(volume, geometry, measured, scan, mask))
        s_, c_ = _loss_terms(volume, geometry, measured, scan, mask)
        t_ = reduce(torch.stack([s_.double(), c_.double()]))
        return float(t_[0] / t_[1].clamp_min(1.0))

    if warm_start is not None:
        with torch.no_grad():
            l_nom = loss_of(nominal)
            start = [g + d.to(g) for g, d in zip(nominal, warm_start)]
            l_warm = loss_of(start)
        accepted = l_warm <= l_nom
        if accepted:
            delta = [d.detach().to(g).clone() for g, d in zip(nominal, warm_start)]
    for d in delta:
        d.requires_grad_(True)
    opt = torch.optim.Adam([{"params": [d], "lr": lr[name]}
                            for d, name in zip(delta, GEOMETRY_NAMES)], betas=tuple(betas))
    sched = torch.optim.lr_scheduler.LambdaLR(
        opt, lambda it: (final_lr_fraction + (1.0 - final_lr_fraction) * 0.5 *
                         (1.0 + math.cos(math.pi * min(it, iterations) / max(iterations, 1)))) *
        lr_gamma ** max(0, it - decay_start) *
        (min(1.0, (it + 1) / warmup_iterations) if warmup_iterations else 1.0))
    if points is None and true_geometry is not None:
        points = lattice_points(volume.shape, scan.voxel_size, scan.volume_offset,
                                device=volume.device)
    result = CalibrationResult(delta=delta, geometry=nominal, warm_start_accepted=accepted)

    def record(it, loss_value):
        entry = {"iteration": it, "loss": loss_value, "time_s": time.perf_counter() - t0}
        if true_geometry is not None:
            geom = [g + d.detach() for g, d in zip(nominal, delta)]
            if reduce is None:
                entry["reproj_px"] = reprojection_error(geom, true_geometry, points,
                                                        scan.pixel_size)
                entry["angle_err_deg"] = angle_error_deg(geom, true_geometry)
            else:
                m = reduce(_metric_terms(geom, true_geometry, points, scan.pixel_size))
                entry["reproj_px"] = float((m[0] / m[1]).sqrt())
                entry["angle_err_deg"] = float((m[2] / m[3]).sqrt())
            ok = entry["reproj_px"] <= target_px and (
                target_angle_deg is None or entry["angle_err_deg"] <= target_angle_deg)
            if ok and result.time_to_target_s is None:
                result.time_to_target_s = entry["time_s"]
                result.iterations_to_target = it
        result.history.append(entry)
        if log_every and it % log_every == 0:
            print({k: (round(v, 5) if isinstance(v, float) else v) for k, v in entry.items()})

    if reduce is None:
        denom = float(measured.numel() if mask is None else mask.sum().clamp_min(1.0))
    else:
        count = float(measured.numel()) if mask is None else mask.double().sum()
        count = torch.as_tensor(count, dtype=torch.float64, device=measured.device).reshape(1)
        denom = float(reduce(count).clamp_min(1.0))
    record(0, float("nan"))
    for it in range(1, iterations + 1):
        opt.zero_grad(set_to_none=True)
        geom = [g + d for g, d in zip(nominal, delta)]
        if fused:
            loss = _fused_loss(volume, geom, measured, scan, mask, denom)
        elif reduce is None:
            loss = _loss(volume, geom, measured, scan, mask)
        else:
            loss = _loss_terms(volume, geom, measured, scan, mask)[0] / denom
        loss.backward()
        opt.step()
        sched.step()
        lv = loss.detach()
        record(it, float(lv) if reduce is None else float(reduce(lv.double().reshape(1))))
        if stop_at_target and result.time_to_target_s is not None:
            break
    result.geometry = [g + d.detach() for g, d in zip(nominal, delta)]
    with torch.no_grad():
        result.final_loss = loss_of(result.geometry)
    return result
