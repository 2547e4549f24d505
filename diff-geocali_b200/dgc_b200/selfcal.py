"""Self-calibration of per-view geometry by image-entropy minimisation.

The reference names a two-stage entropy self-calibration pipeline but does not
ship it (README.md:8; docs/SOURCE.md lists
``selfsupervised_calibration_entropy_2stage.py`` of the original project as
the source of its backprojector's autograd wrapper only).  Unlike
``calibration.calibrate``, which needs the volume, this needs only the
measured projections: a wrong geometry blurs and doubles the FDK
reconstruction, which raises the entropy of its intensity distribution, so
geometry is adjusted to make the reconstruction sharp.

Each iteration: FDK-filtered projections (filtered once, with the nominal
sid/sod, or every iteration with the current ones: ``refilter``) are
backprojected through ``nominal + delta`` (``backproject``, whose
hand-written backward gives the eight per-view geometry gradients), scaled by
pi/A, and the Shannon entropy of the normalised absolute intensities is
minimised with Adam.  Stage 1 fits one offset per geometry family shared by
all views (the well-determined, strongly blurring errors: a detector or
source shift common to the scan); stage 2 then fits per-view offsets.  The
parameter families of each stage are a choice of the caller; the default,
the detector centre in both stages, is what the entropy determines well --
a shared sid or per-view angles moved the estimate away from the truth in
the tests that chose it (the reconstruction's sharpness does not pin the
magnification), and per-view fits drift again after ~40 iterations.
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import torch

from .calibration import GEOMETRY_NAMES, angle_error_deg, reprojection_error
from .filtering import fdk_filter, preweight_frame
from .operator import backproject


def image_entropy(volume, eps=1e-12):
    """Shannon entropy of ``p = |v| / sum |v|`` over the voxels (nats)."""
    a = volume.abs()
    p = a / a.sum().clamp_min(eps)
    return -(p * torch.log(p + eps)).sum()


@dataclass
class SelfCalibrationResult:
    delta: list
    geometry: list
    history: list = field(default_factory=list)


# Adam step sizes per family (radians, length units, pixels), per iteration
DEFAULT_STEP = {"angles": 1e-3, "sid": 1.0, "sod": 1.0, "det_u0": 0.1, "det_v0": 0.1,
                "src_x": 0.1, "src_y": 0.1, "src_z": 0.1}


def entropy_calibrate(projections, nominal, pixel_size, volume_shape, voxel_size,
                      volume_offset=(0.0, 0.0, 0.0),
                      stages=(("det_u0", "det_v0"), ("det_u0", "det_v0")), iterations=(40, 40),
                      lr=None, alpha=0.8, true_geometry=None, points=None, log_every=0,
                      refilter=False, offset_preweight=False):
    """Two-stage entropy self-calibration; returns a ``SelfCalibrationResult``.

    ``stages[0]`` lists the families fitted with one offset shared by all
    views, ``stages[1]`` those fitted per view (starting from stage 1's
    result); ``iterations`` gives each stage's Adam iterations.  With
    ``true_geometry`` (and optionally ``points``) the RMS reprojection error
    [pixels] and angle error are recorded every iteration.  ``refilter``
    filters the projections every iteration with the current sid / sod, so
    that the entropy's gradient reaches those distances through the filter
    too (the whole FDK differentiated; ``fdk_filter``'s own backward).
    ``offset_preweight`` takes the filter's cosine preweight in each view's
    ``preweight_frame`` (the current geometry's with ``refilter``, so that the
    gradient also reaches the detector centres and source offsets through the
    weights; the nominal one otherwise).
    """
    t0 = time.perf_counter()
    step = dict(DEFAULT_STEP, **(lr or {}))
    nominal = [g.detach() for g in nominal]
    A = nominal[0].numel()
    def frame_of(geometry):
        return preweight_frame(*geometry, pixel_size) if offset_preweight else None

    with torch.no_grad():
        filtered = fdk_filter(projections.detach(), pixel_size, nominal[2], nominal[1], alpha,
                              frame=frame_of(nominal))
    scale = math.pi / A
    delta = [torch.zeros_like(g) for g in nominal]
    result = SelfCalibrationResult(delta=delta, geometry=nominal)
    idx = {n: i for i, n in enumerate(GEOMETRY_NAMES)}

    def record(stage, it, loss):
        entry = {"stage": stage, "iteration": it, "entropy": loss,
                 "time_s": time.perf_counter() - t0}
        if true_geometry is not None:
            geom = [g + d for g, d in zip(nominal, delta)]
            if points is not None:
                entry["reproj_px"] = reprojection_error(geom, true_geometry, points, pixel_size)
            entry["angle_err_deg"] = angle_error_deg(geom, true_geometry)
        result.history.append(entry)
        if log_every and it % log_every == 0:
            print(entry)

    for stage, (families, n_it) in enumerate(zip(stages, iterations)):
        shared = stage == 0
        params = {}
        for name in families:
            k = idx[name]
            params[name] = (torch.zeros(1, device=nominal[k].device, requires_grad=True)
                            if shared else delta[k].clone().requires_grad_(True))
        opt = torch.optim.Adam([{"params": [p], "lr": step[n]} for n, p in params.items()],
                               betas=(0.9, 0.99))
        record(stage, 0, float("nan"))
        for it in range(1, n_it + 1):
            opt.zero_grad(set_to_none=True)
            geom = []
            for k, (g, d) in enumerate(zip(nominal, delta)):
                name = GEOMETRY_NAMES[k]
                if name in params:
                    geom.append(g + d + params[name] if shared else g + params[name])
                else:
                    geom.append(g + d)
            filt = (fdk_filter(projections.detach(), pixel_size, geom[2], geom[1], alpha,
                               frame=frame_of(geom)) if refilter else filtered)
            vol = backproject(filt, *geom, pixel_size, volume_shape, voxel_size,
                              volume_offset) * scale
            loss = image_entropy(vol)
            loss.backward()
            opt.step()
            with torch.no_grad():
                for name, p in params.items():
                    k = idx[name]
                    if shared:
                        delta[k] += p.detach()
                        p.zero_()
                    else:
                        delta[k].copy_(p.detach())
            record(stage, it, float(loss.detach()))
    result.geometry = [g + d for g, d in zip(nominal, delta)]
    return result


__all__ = ["entropy_calibrate", "image_entropy", "SelfCalibrationResult", "DEFAULT_STEP"]
